"""Known-answer cases for the beamformer, sized to cross source tiles, warps
and time tiles of the staged kernel.

Each case states its answer from first principles: a pure shift, exact ties
(lowest source index wins), an injected pulse whose source must win, all-zero
weights and delays past the record.  The CPU tests pin every answer against
the oracle; the GPU tests run the same cases through the drop-in symbols
(beamform / beamform_max, the reference's argument order) and compare bit
for bit with the answer and the oracle.
"""
import numpy as np
import pytest

from test_gpu_parity import bits, dropin_max, dropin_none


def case_pure_shift():
    """One station, one phase, unit weights: source i's beam is the trace
    shifted by its delay i % 37 (strict: samples whose shifted index leaves
    the record are not computed).  The trace increases, so at each sample
    the largest valid delay wins, its lowest source index among equals."""
    T, N = 1000, 200
    U = (np.arange(T, dtype=np.float32) * 0.25).reshape(1, T, 1)
    d = (np.arange(N) % 37).astype(np.int32)
    D = d.reshape(N, 1, 1)
    W = np.ones((N, 1), dtype=np.float32)
    beam = np.zeros((N, T), dtype=np.float32)
    for i in range(N):
        beam[i, :T - d[i]] = U[0, d[i]:, 0]
    am = np.zeros(T, dtype=np.int32)
    bm = np.zeros(T, dtype=np.float32)
    for t in range(T):
        ok = np.nonzero(t + d < T)[0]
        best = ok[np.argmax(d[ok])]  # first index among the largest valid delays
        am[t], bm[t] = best, U[0, t + d[best], 0]
    return U, D, W, {"beam": beam, "max": (bm, am)}


def case_exact_ties():
    """300 sources in 5 groups of identical delays and weights, the group of
    source i being (7 i) mod 5, so equal beams sit in different tiles and
    warps.  Where a group wins, the answer is its lowest source index."""
    rng = np.random.default_rng(3)
    T, N, S, P = 700, 300, 6, 2
    U = rng.standard_normal((S, T, P)).astype(np.float32)
    gd = rng.integers(0, 60, size=(5, S, P)).astype(np.int32)
    gw = rng.uniform(0.5, 1.5, size=(5, S)).astype(np.float32)
    g = (7 * np.arange(N)) % 5
    D, W = gd[g], gw[g]
    first = np.array([np.min(np.nonzero(g == k)[0]) for k in range(5)])
    return U, D, W, {"group_first": first, "group": g}


def case_injected_pulse():
    """Noise plus a Gaussian pulse placed at t0 + delay(j, s, p) on every
    station and phase: source j's beam peaks at t0 and wins there."""
    rng = np.random.default_rng(4)
    T, N, S, P, j, t0 = 2000, 500, 10, 2, 317, 900
    D = rng.integers(0, 300, size=(N, S, P)).astype(np.int32)
    W = np.ones((N, S), dtype=np.float32)
    U = (0.05 * np.abs(rng.standard_normal((S, T, P)))).astype(np.float32)
    tt = np.arange(T)
    for s in range(S):
        for p in range(P):
            U[s, :, p] += np.exp(-0.5 * ((tt - t0 - D[j, s, p]) / 4.0) ** 2).astype(np.float32)
    return U, D, W, {"source": j, "t0": t0}


def case_no_candidates():
    """All-zero weights (strict: no source is valid, so beam_max keeps the
    caller's content and argmax is 0; flexible: every source competes with a
    beam of 0), and delays past the record (strict: no candidate; flexible:
    every term skipped, so every beam is 0)."""
    rng = np.random.default_rng(5)
    T, N, S, P = 300, 130, 4, 2
    U = rng.standard_normal((S, T, P)).astype(np.float32)
    D0 = rng.integers(0, 20, size=(N, S, P)).astype(np.int32)
    W0 = np.zeros((N, S), dtype=np.float32)
    D1 = (T + rng.integers(0, 50, size=(N, S, P))).astype(np.int32)
    W1 = np.ones((N, S), dtype=np.float32)
    return U, (D0, W0), (D1, W1)


# ---- the answers against the oracle (CPU) ---------------------------------

def test_pure_shift_answer_matches_oracle(oracle_lib):
    U, D, W, ans = case_pure_shift()
    assert np.array_equal(bits(oracle_lib.beamform(U, D, W, 0)), bits(ans["beam"]))
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert np.array_equal(bits(bm), bits(ans["max"][0])) and np.array_equal(am, ans["max"][1])


def test_tie_answer_matches_oracle(oracle_lib):
    U, D, W, ans = case_exact_ties()
    for oob in (0, 1):
        bm, am = oracle_lib.beamform_max(U, D, W, oob)
        has = np.isin(am, ans["group_first"])
        assert has.mean() > 0.9
        assert np.array_equal(am[has], ans["group_first"][ans["group"][am[has]]])


def test_pulse_answer_matches_oracle(oracle_lib):
    U, D, W, ans = case_injected_pulse()
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert am[ans["t0"]] == ans["source"]


def test_no_candidate_answer_matches_oracle(oracle_lib):
    U, (D0, W0), (D1, W1) = case_no_candidates()
    for oob in (0, 1):
        bm, am = oracle_lib.beamform_max(U, D0, W0, oob)
        assert np.all(bm == 0) and np.all(am == 0)
    bm, am = oracle_lib.beamform_max(U, D1, W1, 0)
    assert np.all(bm == 0) and np.all(am == 0)
    assert np.all(oracle_lib.beamform(U, D1, W1, 1) == 0)


# ---- the same cases on the GPU ---------------------------------------------

@pytest.mark.gpu
def test_pure_shift_on_gpu(cuda, bplib):
    U, D, W, ans = case_pure_shift()
    beam = dropin_none(bplib, U, D, W, 0)
    assert np.array_equal(bits(beam), bits(ans["beam"]))
    bm, am = dropin_max(bplib, U, D, W, 0)
    assert np.array_equal(bits(bm), bits(ans["max"][0])) and np.array_equal(am, ans["max"][1])


@pytest.mark.gpu
def test_exact_ties_lowest_index_on_gpu(cuda, bplib, oracle_lib):
    U, D, W, ans = case_exact_ties()
    for oob in (0, 1):
        bm, am = dropin_max(bplib, U, D, W, oob)
        obm, oam = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam), oob
        # every sample's winner is the first source of its group
        assert np.array_equal(am, ans["group_first"][ans["group"][am]]), oob


@pytest.mark.gpu
def test_injected_pulse_wins_on_gpu(cuda, bplib, oracle_lib):
    U, D, W, ans = case_injected_pulse()
    bm, am = dropin_max(bplib, U, D, W, 0)
    assert am[ans["t0"]] == ans["source"]
    obm, oam = oracle_lib.beamform_max(U, D, W, 0)
    assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)


@pytest.mark.gpu
def test_no_candidates_on_gpu(cuda, bplib):
    U, (D0, W0), (D1, W1) = case_no_candidates()
    bm, am = dropin_max(bplib, U, D0, W0, 0, init=-7.0)
    assert np.all(bm == -7.0) and np.all(am == 0)
    bm, am = dropin_max(bplib, U, D0, W0, 1, init=-7.0)
    assert np.all(bm == 0.0) and np.all(am == 0)
    bm, am = dropin_max(bplib, U, D1, W1, 0, init=-7.0)
    assert np.all(bm == -7.0) and np.all(am == 0)
    bm, am = dropin_max(bplib, U, D1, W1, 1, init=-7.0)
    assert np.all(bm == 0.0) and np.all(am == 0)
    assert np.all(dropin_none(bplib, U, D1, W1, 1, init=-7.0) == 0.0)
