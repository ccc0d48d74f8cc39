"""bench.py's host-side arithmetic on the CPU: the effective-term count that
the roofline's achieved rate divides (checked against a brute-force count of
the terms the reference computes), and the clock-record summary that decides
whether a run is kept."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def brute_force_terms(D, W, T, flexible):
    """(source, sample, station, phase) terms the reference evaluates
    (beampower/src/beamform.c:49-105 under the rule of :276-306)."""
    N, S, P = D.shape
    total = 0
    for i in range(N):
        weighted = [s for s in range(S) if W[i, s] != 0]
        if not weighted:
            continue
        d = D[i, weighted, :].astype(np.int64)
        for t in range(T):
            if flexible:
                total += int(((t + d >= 0) & (t + d < T)).sum())
            elif t + d.min() >= 0 and t + d.max() < T:
                total += len(weighted) * P
    return total


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("flexible", [False, True])
def test_effective_terms_match_brute_force(seed, flexible):
    rng = np.random.default_rng(seed)
    N, S, P, T = 40, 5, int(rng.integers(1, 4)), int(rng.integers(1, 90))
    D = rng.integers(-T, 2 * T, size=(N, S, P)).astype(np.int32)
    if seed % 2:
        D = rng.integers(-3, T // 3 + 1, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.5, 2.0, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < 0.3] = 0.0
    W[::7] = 0.0  # sources without a weighted station
    assert bench.effective_terms(D, W, T, flexible) == brute_force_terms(D, W, T, flexible)


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.proc, s.lines = _Proc(), lines
    return s


def test_clock_summary_median_max_and_reasons():
    rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1900, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
            "garbage line",
            "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    out = _sampler(rows).stop()
    assert out == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                   "samples": 3}


def test_clock_summary_flags_thermal_and_empty_record():
    rows = ["0, 1500, 1965, 900.0, 0x40, Active, Not Active, Active, Not Active"]
    assert _sampler(rows).stop()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert _sampler([]).stop() is None
    assert bench.ClockSampler(0).stop() is None  # nvidia-smi never started

