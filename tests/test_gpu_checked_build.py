"""The index-checked build (libbeampower_b200_checked.so, BP_DEBUG_CHECKS):
the staged kernel checks every bulk copy and every shared-memory read and
records a failure in its status word instead of faulting.  Parity cases,
every storage and both rules, and a persistent batch run through it in a
child process (tests/_checked_build_run.py) with no check failing and the
FP32 results equal to the reference fixtures."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_checked_build_runs_clean(cuda):
    lib = os.path.join(ROOT, "beampower_b200", "lib", "libbeampower_b200_checked.so")
    assert os.path.exists(lib), "build it with: python -m beampower_b200.build --checked"
    env = dict(os.environ, BEAMPOWER_B200_LIBRARY=lib)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "_checked_build_run.py")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "CHECKED OK" in r.stdout
