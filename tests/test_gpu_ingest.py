"""Travel-time conversion on the GPU: identical integers to the tutorial's
``sec_to_samp`` (fixtures) and to the oracle at the size of the 400,000
source x 60 station x 2 phase grid; a table built from seconds equals one
built from the converted delays."""
import numpy as np
import pytest

from test_ingest_oracle import load_ingest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sr", [25, 100])
def test_matches_tutorial_fixtures(cuda, sr):
    from beampower_b200.ingest import sec_to_samp
    g = load_ingest()
    assert np.array_equal(sec_to_samp(g["seconds"], float(sr)), g[f"delays_{sr}"])
    assert np.array_equal(sec_to_samp(g["seconds"], float(sr), relative=True),
                          g[f"relative_{sr}"])


def test_full_grid_against_oracle(cuda):
    import torch
    from oracle import ingest as oing
    from beampower_b200.ingest import sec_to_samp
    rng = np.random.default_rng(1)
    tt = rng.uniform(0.0, 40.0, size=(400000, 60, 2)).astype(np.float32)
    got = sec_to_samp(torch.from_numpy(tt).to(cuda), 50.0, relative=True)
    assert got.dtype == torch.int32 and got.is_cuda
    assert np.array_equal(got.cpu().numpy(), oing.sec_to_samp(tt, 50.0, relative=True))


def test_table_from_travel_times(cuda):
    import torch
    from oracle import ingest as oing
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(2)
    tt = rng.uniform(0.0, 10.0, size=(700, 9, 2)).astype(np.float32)
    W = rng.uniform(0.5, 1.5, size=(700, 9)).astype(np.float32)
    a = TravelTimeTable.from_travel_times(tt, 25.0, W, relative=True)
    assert np.array_equal(a.delays.cpu().numpy(), oing.sec_to_samp(tt, 25.0, relative=True))
    a.close()
