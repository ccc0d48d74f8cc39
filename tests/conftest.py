"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
the CPU.  The CPU oracle (oracle/) is only ever used here as the checker."""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_oracle():
    from oracle import oracle as orc
    if not os.path.exists(orc.ORACLE_SO):
        orc.build(reference_root=None)
    return orc


@pytest.fixture(scope="session")
def orc():
    return _ensure_oracle()


@pytest.fixture(scope="session")
def oracle_lib(orc):
    return orc.Oracle()


def golden_small_names():
    return sorted(os.path.basename(p)[len("small_"):-len(".npz")]
                  for p in glob.glob(os.path.join(GOLDEN, "small_*.npz")))


def load_golden(name):
    with np.load(os.path.join(GOLDEN, f"small_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests error out (not skip) when there is none."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def bplib():
    import beampower_b200
    return beampower_b200.load_library("gpu")
