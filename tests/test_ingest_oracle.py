"""CPU check of the travel-time conversion oracle (oracle/ingest.py)
against fixtures made from the reference tutorial's own ``sec_to_samp``
(tests/golden/make_ingest_golden.py): identical integers."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

from oracle import ingest as oing


def load_ingest():
    with np.load(os.path.join(GOLDEN, "ingest.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("sr", [25, 100])
def test_oracle_matches_tutorial(sr):
    g = load_ingest()
    assert np.array_equal(oing.sec_to_samp(g["seconds"], float(sr)), g[f"delays_{sr}"])
    assert np.array_equal(oing.sec_to_samp(g["seconds"], float(sr), relative=True),
                          g[f"relative_{sr}"])
