"""The oracle against the reference's own C library over a seeded sweep of
shapes: sources, stations, channels, phases and samples drawn per case
(including single-sample records, one station, one phase, no sources),
delays reaching past either end of the record, a fifth of the stations
unweighted and non-unit weights.  Every output is compared bit for bit.

The reference library is oracle/_ref/beamform_cpu.so, built from
beampower/src/beamform.c by oracle/Makefile when a reference checkout is
present; without it the sweep is skipped (the committed golden fixtures
still pin the oracle).

Two reference behaviours bound the sweep:
* beamform_max's strict rule tests ``t + min < 0`` on size_t operands
  (beampower/src/beamform.c:281), so a negative minimum delay reads outside
  the trace there; the strict max cases keep every delay non-negative (the
  reduce='none' and flexible cases take negative delays, which the reference
  handles: int time index at beamform.c:194-201, wrap-around caught by the
  upper test at beamform.c:97);
* beamform_differential declares its per-source min / max delay outside the
  OpenMP loop (beamform.c:355) and leaves them out of the loop's private list
  (beamform.c:370, unlike the reduce='none' loop at beamform.c:185), so with
  several threads one source can be tested against another's range
  (beamform.c:377-378); the reference is run with one thread there.
"""
import os

import numpy as np
import pytest

from oracle.oracle import REF_CPU_SO

pytestmark = pytest.mark.skipif(not os.path.exists(REF_CPU_SO),
                                reason="reference CPU library not built (oracle/_ref)")

SEEDS = list(range(32))


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _case(seed, non_negative):
    rng = np.random.default_rng(1000 + seed)
    N = int(rng.choice([0, 1, 2, 7, 33, 150, 300])) if seed % 8 else int(rng.integers(1, 40))
    S = int(rng.integers(1, 10))
    C = int(rng.integers(1, 4))
    P = int(rng.integers(1, 5))
    T = int(rng.choice([1, 2, 5, 64, 257, 700]))
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.0, 1.5, size=(S, C, P)).astype(np.float32)
    A[rng.random(A.shape) < 0.3] = 0.0
    reach = max(T // 2, 2)
    lo = 0 if non_negative else -reach
    D = rng.integers(lo, T + reach, size=(N, S, P)).astype(np.int32)
    if seed % 3 == 0:  # most sources inside the record, as in a real grid
        D = rng.integers(0 if non_negative else -2, max(T // 4, 1) + 1,
                         size=(N, S, P)).astype(np.int32)
    W = np.where(rng.random((N, S)) < 0.5, 1.0,
                 rng.uniform(0.1, 3.0, size=(N, S))).astype(np.float32)
    W[rng.random(W.shape) < 0.2] = 0.0
    return F, A, D, W


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Reference
    return Reference()


@pytest.mark.parametrize("seed", SEEDS)
def test_prestack_and_full_beam_match_reference(oracle_lib, ref, seed):
    F, A, D, W = _case(seed, non_negative=False)
    U_ref = ref.prestack(F, A, num_threads=2)
    U = oracle_lib.prestack(F, A)
    assert np.array_equal(_bits(U), _bits(U_ref))
    for oob in (0, 1):
        want = ref.beamform(U_ref, D, W, oob, num_threads=3)
        got = oracle_lib.beamform(U_ref, D, W, oob)
        assert np.array_equal(_bits(got), _bits(want)), oob


@pytest.mark.parametrize("seed", SEEDS)
def test_max_matches_reference(oracle_lib, ref, seed):
    F, A, D, W = _case(seed, non_negative=True)
    U = ref.prestack(F, A)
    for oob in (0, 1):
        bm_r, am_r = ref.beamform_max(U, D, W, oob, num_threads=3)
        bm, am = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(_bits(bm), _bits(bm_r)), oob
        assert np.array_equal(am, am_r), oob
    # flexible rule with delays on both sides of the record
    _, _, Dn, _ = _case(seed, non_negative=False)
    bm_r, am_r = ref.beamform_max(U, Dn, W, 1, num_threads=3)
    bm, am = oracle_lib.beamform_max(U, Dn, W, 1)
    assert np.array_equal(_bits(bm), _bits(bm_r))
    assert np.array_equal(am, am_r)


@pytest.mark.parametrize("seed", SEEDS)
def test_differential_matches_reference(oracle_lib, ref, seed):
    F, A, D, W = _case(seed, non_negative=False)
    U = ref.prestack(F, A)
    want = ref.beamform_differential(U, D, W, num_threads=1)
    got = oracle_lib.beamform_differential(U, D, W)
    assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("seed", SEEDS)
def test_sampled_max_matches_full_max(oracle_lib, ref, seed):
    """The oracle's max at chosen samples (the checker of the full-size GPU
    tests) equals the reference's max over the whole record at those
    samples, including samples without a candidate (0 and index 0)."""
    F, A, D, W = _case(seed, non_negative=True)
    U = ref.prestack(F, A)
    T = U.shape[1]
    rng = np.random.default_rng(seed)
    times = np.unique(np.concatenate([[0, T - 1], rng.integers(0, T, size=min(T, 25))]))
    for oob in (0, 1):
        bm_r, am_r = ref.beamform_max(U, D, W, oob, num_threads=3)
        bm, am = oracle_lib.beamform_max_at(U, D, W, times, oob)
        assert np.array_equal(_bits(bm), _bits(bm_r[times])), oob
        assert np.array_equal(am, am_r[times]), oob
