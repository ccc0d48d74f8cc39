"""The oracle, pinned: against the golden fixtures made by running the
reference's own C library, against the reference library itself when it is
built here, against float64 restatements, and on known-answer cases."""
import os

import numpy as np
import pytest

from conftest import golden_small_names, load_golden

NAMES = golden_small_names()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(oracle_lib, name):
    g = load_golden(name)
    U = oracle_lib.prestack(g["F"], g["A"])
    assert np.array_equal(bits(U), bits(g["U"]))
    for oob, tag in ((0, "strict"), (1, "flexible")):
        if f"beam_max_{tag}" in g:
            bm, am = oracle_lib.beamform_max(g["U"], g["D"], g["W"], oob)
            assert np.array_equal(bits(bm), bits(g[f"beam_max_{tag}"])), tag
            assert np.array_equal(am, g[f"argmax_{tag}"]), tag
        beam = oracle_lib.beamform(g["U"], g["D"], g["W"], oob)
        assert np.array_equal(bits(beam), bits(g[f"beam_{tag}"])), tag
    diff = oracle_lib.beamform_differential(g["U"], g["D"], g["W"])
    assert np.array_equal(bits(diff), bits(g["differential"]))


def test_oracle_matches_reference_tutorial_scale(oracle_lib):
    from beampower_b200.synthetic import SMALL, digest, make_workload
    with np.load(os.path.join(os.path.dirname(__file__), "golden", "tutorial_scale.npz")) as z:
        g = {k: z[k] for k in z.files}
    wl = make_workload(SMALL)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    assert digest(F, A, D, W) == str(g["digest"]), "synthetic generator drifted"
    U = oracle_lib.prestack(F, A)
    assert digest(U) == str(g["U_digest"])
    for oob, tag in ((0, "strict"), (1, "flexible")):
        bm, am = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(g[f"beam_max_{tag}"]))
        assert np.array_equal(am, g[f"argmax_{tag}"])
    # the injected events are found at their sources
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    for src, t0 in wl["events"]:
        assert am[t0] == src


@pytest.mark.parametrize("name", ["random_p2", "long_delays", "negative_delays"])
def test_oracle_within_fp64(oracle_lib, orc, name):
    g = load_golden(name)
    ref64, valid = orc.fp64_beams(orc.fp64_prestack(g["F"], g["A"]), g["D"], g["W"], 1)
    beam = oracle_lib.beamform(g["U"], g["D"], g["W"], 1)
    scale = np.maximum(np.abs(ref64), 1e-30)
    rel = np.abs(beam - ref64) / scale
    assert np.nanmax(rel[np.abs(ref64) > 1e-3]) < 1e-5


def test_oracle_strict_rule_with_negative_delays(oracle_lib, orc):
    """Strict rule: computed iff 0 <= t + min and t + max < T (weighted)."""
    g = load_golden("negative_delays")
    beam = np.full((g["D"].shape[0], g["U"].shape[1]), -7.0, dtype=np.float32)
    beam = oracle_lib.beamform(g["U"], g["D"], g["W"], 0, out=beam)
    _, valid = orc.fp64_beams(g["U"], g["D"], g["W"], 0)
    assert np.all((beam != -7.0) == valid)
    # the reference's reduce='none' agrees (int time index, beamform.c:194)
    assert np.array_equal(bits(np.where(valid, beam, 0)), bits(g["beam_strict"]))
    bm, am = oracle_lib.beamform_max(g["U"], g["D"], g["W"], 0)
    full = np.where(valid, beam, -np.inf)
    has = valid.any(axis=0)
    assert np.array_equal(am[has], np.argmax(full, axis=0)[has])
    assert np.array_equal(bits(bm[has]), bits(full.max(axis=0)[has]))
    assert np.all(bm[~has] == 0) and np.all(am[~has] == 0)


def test_known_answer_pure_shift(oracle_lib):
    """One station, one phase, unit weight: the beam is the shifted trace."""
    T = 200
    U = np.arange(T, dtype=np.float32).reshape(1, T, 1) * 0.5
    D = np.array([[[7]], [[0]], [[30]]], dtype=np.int32)
    W = np.ones((3, 1), dtype=np.float32)
    beam = oracle_lib.beamform(U, D, W, 0)
    for i, d in enumerate(D[:, 0, 0]):
        assert np.array_equal(beam[i, :T - d], U[0, d:, 0])
        assert np.all(beam[i, T - d:] == 0)
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    # increasing trace: the largest shift wins while it is valid
    assert np.all(am[:T - 30] == 2)


def test_known_answer_ties_and_all_negative(oracle_lib):
    T = 50
    U = -np.ones((2, T, 1), dtype=np.float32)
    D = np.zeros((4, 2, 1), dtype=np.int32)
    W = np.ones((4, 2), dtype=np.float32)
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert np.all(bm == -2.0) and np.all(am == 0)       # negative beams are legal
    W[0] = 0.0                                            # source 0 never valid (strict)
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert np.all(am == 1)
    bm, am = oracle_lib.beamform_max(U, D, W, 1)          # flexible: 0.0 competes
    assert np.all(am == 0) and np.all(bm == 0.0)
    W[:] = 0.0
    bm, am = oracle_lib.beamform_max(U, D, W, 0)          # nothing computed
    assert np.all(bm == 0.0) and np.all(am == 0)


def test_known_answer_nan_never_wins(oracle_lib):
    T = 20
    U = np.ones((1, T, 1), dtype=np.float32)
    U[0, 5] = np.nan
    D = np.zeros((2, 1, 1), dtype=np.int32)
    W = np.array([[1.0], [0.5]], dtype=np.float32)
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert am[5] == 0 and bm[5] == 0.0                    # NaN beams are not candidates
    assert np.all(am[np.arange(T) != 5] == 0)


def test_reference_gpu_build_exports_its_symbols():
    """The reference's CUDA path built for sm_100a (oracle/_ref, the timed
    "plain GPU path" baseline) loads without a GPU and exports the two
    symbols beampower/core.py:65-87 binds."""
    import ctypes as ct
    from oracle.oracle import REF_GPU_SO
    if not os.path.exists(REF_GPU_SO):
        pytest.skip("reference GPU library not built (oracle/_ref)")
    lib = ct.CDLL(REF_GPU_SO)
    assert hasattr(lib, "beamform") and hasattr(lib, "beamform_max")
