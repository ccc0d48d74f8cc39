"""The host-buffer path for many sources (reduce='max', at least 2 x 65,536
sources) runs as a pipeline over source chunks: each chunk's delays and
weights upload while the previous chunk's kernel runs, one table per chunk
with source indexes offset by the chunk's start.  The result must be the
single call's, bit for bit: checked against the oracle and against the
device path on one table, with the staged kernel and with the direct kernel
(delay windows too wide for the staged kernel's shared-memory ring: eight
stations of independent random delays over 36,000 samples, which no tiling
can make compact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return np.where(np.isnan(a), np.uint32(0x7FC00000), a.view(np.uint32))


def _case(seed, N, S, C, P, T, dmax):
    rng = np.random.default_rng(seed)
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, dmax + 1, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.5, 1.5, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < 0.2] = 0.0
    return F, A, D, W


@pytest.mark.parametrize("oob", ["strict", "flexible"])
@pytest.mark.parametrize("wide", [False, True])
def test_chunked_host_path_equals_single_table(cuda, oracle_lib, oob, wide):
    import torch
    import beampower_b200 as bp
    from beampower_b200.tables import TravelTimeTable
    if wide:  # windows beyond the ring: every chunk table runs the direct kernel
        F, A, D, W = _case(7, 140_000, 8, 2, 1, 40_000, 36_000)
    else:
        F, A, D, W = _case(8, 150_000, 6, 3, 2, 3_000, 400)
    flag = 0 if oob == "strict" else 1
    bm, am = bp.beamform(F, D, A, W, reduce="max", out_of_bounds=oob)
    table = TravelTimeTable(D, W)
    assert bool(table.info["uses_window_kernel"]) == (not wide)
    tr = table.traces_from_features(F, A, storage="fp32")
    dbm, dam = table.beamform_max(tr, flag)
    torch.cuda.synchronize()
    assert np.array_equal(bits(bm), bits(dbm.cpu().numpy()))
    assert np.array_equal(am, dam.cpu().numpy())
    obm, oam = oracle_lib.beamform_max(oracle_lib.prestack(F, A), D, W, flag)
    assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)
    table.close()
