"""GPU parity: the sm_100a kernels, called through the C-ABI, against the
golden fixtures made by the reference's own C library and against the oracle.

FP32 storage is bit-exact: same valid-sample mask, same beam bits, same
argmax (the kernels keep the reference's per-(source, sample) order of
rounded multiplies and adds).  Where the reference's strict reduce='max' is
undefined (negative delays) the oracle's documented rule is the target.
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import golden_small_names, load_golden

pytestmark = pytest.mark.gpu
NAMES = golden_small_names()


def bits(a):
    """float32 bit patterns, with every NaN mapped to one pattern: the GPU
    returns the canonical NaN where x86 propagates the input's payload, and
    the reference semantics only say "NaN" (it never wins a max)."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    return np.where(np.isnan(a), np.uint32(0x7FC00000), a.view(np.uint32))


def _fp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


def _ip(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_int))


def dropin_max(lib, U, D, W, oob, init=0.0):
    """The reference's GPU symbol beamform_max, reference argument order."""
    U = np.ascontiguousarray(U, np.float32)
    D = np.ascontiguousarray(D, np.int32)
    W = np.ascontiguousarray(W, np.float32)
    S, T, P = U.shape
    N = D.shape[0]
    bm = np.full(T, init, dtype=np.float32)
    am = np.full(T, -5, dtype=np.int32)
    rc = lib.beamform_max(_fp(U), _ip(D), _fp(W), T, N, S, P, int(oob), _fp(bm), _ip(am))
    assert rc == 0, lib.bp_last_error()
    return bm, am


def dropin_none(lib, U, D, W, oob, init=0.0):
    U = np.ascontiguousarray(U, np.float32)
    D = np.ascontiguousarray(D, np.int32)
    W = np.ascontiguousarray(W, np.float32)
    S, T, P = U.shape
    N = D.shape[0]
    beam = np.full((N, T), init, dtype=np.float32)
    rc = lib.beamform(_fp(U), _ip(D), _fp(W), T, N, S, P, int(oob), _fp(beam))
    assert rc == 0, lib.bp_last_error()
    return beam


@pytest.mark.parametrize("name", NAMES)
def test_dropin_beamform_max_matches_reference(cuda, bplib, name):
    g = load_golden(name)
    for oob, tag in ((0, "strict"), (1, "flexible")):
        if f"beam_max_{tag}" not in g:
            continue
        bm, am = dropin_max(bplib, g["U"], g["D"], g["W"], oob)
        assert np.array_equal(bits(bm), bits(g[f"beam_max_{tag}"])), tag
        assert np.array_equal(am, g[f"argmax_{tag}"]), tag


@pytest.mark.parametrize("name", NAMES)
def test_dropin_beamform_none_matches_reference(cuda, bplib, name):
    g = load_golden(name)
    for oob, tag in ((0, "strict"), (1, "flexible")):
        beam = dropin_none(bplib, g["U"], g["D"], g["W"], oob)
        assert np.array_equal(bits(beam), bits(g[f"beam_{tag}"])), tag


@pytest.mark.parametrize("name", NAMES)
def test_frontend_numpy_matches_reference(cuda, name):
    """beampower_b200.beamform on raw features (GPU prestack included)."""
    import beampower_b200 as bp
    g = load_golden(name)
    for oob, tag in ((0, "strict"), (1, "flexible")):
        if f"beam_max_{tag}" in g:
            bm, am = bp.beamform(g["F"], g["D"], g["A"], g["W"], device="gpu", reduce="max",
                                 out_of_bounds=tag)
            assert bm.dtype == np.float32 and am.dtype == np.int32
            assert np.array_equal(bits(bm), bits(g[f"beam_max_{tag}"])), tag
            assert np.array_equal(am, g[f"argmax_{tag}"]), tag
        beam = bp.beamform(g["F"], g["D"], g["A"], g["W"], device="gpu", reduce=None,
                           out_of_bounds=tag)
        assert beam.shape == g[f"beam_{tag}"].shape
        assert np.array_equal(bits(beam), bits(g[f"beam_{tag}"])), tag


@pytest.mark.parametrize("name", NAMES)
def test_prestack_and_differential_match_reference(cuda, name):
    import beampower_b200 as bp
    g = load_golden(name)
    U = bp.prestack_traces(g["F"], g["A"])
    assert np.array_equal(bits(U), bits(g["U"]))
    beam = bp.beamform(g["F"], g["D"], g["A"], g["W"], mode="differential", reduce=None)
    assert np.array_equal(bits(beam), bits(g["differential"]))


def test_negative_delays_strict_max_follows_rule(cuda, bplib, oracle_lib):
    g = load_golden("negative_delays")
    bm, am = dropin_max(bplib, g["U"], g["D"], g["W"], 0)
    obm, oam = oracle_lib.beamform_max(g["U"], g["D"], g["W"], 0)
    assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)


def test_untouched_outputs_keep_caller_content(cuda, bplib, oracle_lib, orc):
    """beam_max keeps the caller's value where no source is a candidate, and
    strict reduce='none' leaves invalid entries alone."""
    g = load_golden("long_delays")
    _, valid = orc.fp64_beams(g["U"], g["D"], g["W"], 0)
    has = valid.any(axis=0)
    assert (~has).any() and has.any()
    bm, am = dropin_max(bplib, g["U"], g["D"], g["W"], 0, init=-3.5)
    assert np.all(bm[~has] == -3.5) and np.all(am[~has] == 0)
    assert np.array_equal(bits(bm[has]), bits(g["beam_max_strict"][has]))
    assert np.array_equal(am, g["argmax_strict"])
    beam = dropin_none(bplib, g["U"], g["D"], g["W"], 0, init=9.0)
    obeam = oracle_lib.beamform(g["U"], g["D"], g["W"], 0,
                                out=np.full_like(beam, 9.0))
    assert np.array_equal(bits(beam), bits(obeam))


def test_tutorial_scale_matches_reference(cuda):
    """The 4,000-source network: numpy front-end, bit-exact vs the reference."""
    import os
    import beampower_b200 as bp
    from beampower_b200.synthetic import SMALL, digest, make_workload
    with np.load(os.path.join(os.path.dirname(__file__), "golden", "tutorial_scale.npz")) as z:
        gold = {k: z[k] for k in z.files}
    wl = make_workload(SMALL)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    assert digest(F, A, D, W) == str(gold["digest"])
    for tag in ("strict", "flexible"):
        bm, am = bp.beamform(F, D, A, W, device="gpu", reduce="max", out_of_bounds=tag)
        assert np.array_equal(bits(bm), bits(gold[f"beam_max_{tag}"])), tag
        assert np.array_equal(am, gold[f"argmax_{tag}"]), tag
    for src, t0 in wl["events"]:
        assert am[t0] == src


def test_torch_tensor_path(cuda):
    import torch
    import beampower_b200 as bp
    g = load_golden("random_p2")
    dev = torch.device("cuda", 0)
    args = [torch.from_numpy(g[k]).to(dev) for k in ("F", "D", "A", "W")]
    bm, am = bp.beamform(*args, reduce="max", out_of_bounds="strict")
    assert bm.is_cuda and am.dtype == torch.int32
    assert np.array_equal(bits(bm.cpu().numpy()), bits(g["beam_max_strict"]))
    assert np.array_equal(am.cpu().numpy(), g["argmax_strict"])
    beam = bp.beamform(*args, reduce=None, out_of_bounds="flexible")
    assert np.array_equal(bits(beam.cpu().numpy()), bits(g["beam_flexible"]))


def _random_problem(rng, N, S, P, T, dmax, dmin=0, zero_frac=0.2, C=3):
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.0, 1.5, size=(S, C, P)).astype(np.float32)
    D = rng.integers(dmin, dmax + 1, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.25, 2.0, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < zero_frac] = 0.0
    return F, A, D, W


@pytest.mark.parametrize("N,S,P,T,dmax", [
    (1, 1, 1, 1, 0),          # smallest problem
    (65, 3, 2, 255, 40),      # one source past a tile, T below one time tile
    (64, 9, 2, 257, 300),     # T just past one time tile, delays > T
    (130, 4, 1, 1000, 700),   # P = 1
    (100, 5, 3, 777, 120),    # P = 3
    (70, 4, 4, 512, 64),      # P = 4
    (50, 3, 6, 300, 50),      # P = 6: direct kernel
])
def test_shapes_against_oracle(cuda, bplib, oracle_lib, N, S, P, T, dmax):
    rng = np.random.default_rng(N * 7 + S * 3 + P + T)
    F, A, D, W = _random_problem(rng, N, S, P, T, dmax)
    U = oracle_lib.prestack(F, A)
    for oob in (0, 1):
        bm, am = dropin_max(bplib, U, D, W, oob)
        obm, oam = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(obm)), oob
        assert np.array_equal(am, oam), oob
        beam = dropin_none(bplib, U, D, W, oob)
        assert np.array_equal(bits(beam), bits(oracle_lib.beamform(U, D, W, oob))), oob


def test_wide_delay_spread_uses_direct_kernel(cuda, bplib, oracle_lib):
    """Delay windows too wide for shared memory: the table falls back to the
    direct kernel, results stay exact."""
    import torch
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(5)
    F, A, D, W = _random_problem(rng, 80, 4, 2, 3000, 90000, zero_frac=0.0)
    table = TravelTimeTable(D, W)
    assert table.info["uses_window_kernel"] == 0
    U = oracle_lib.prestack(F, A)
    for oob in (0, 1):
        bm, am = dropin_max(bplib, U, D, W, oob)
        obm, oam = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)
    table.close()
    torch.cuda.synchronize()


def test_nonfinite_weights_flexible(cuda, bplib, oracle_lib):
    """Inf / NaN weights with out-of-range terms: the checked kernel variant
    skips those terms exactly like the reference."""
    rng = np.random.default_rng(11)
    F, A, D, W = _random_problem(rng, 90, 5, 2, 400, 300, zero_frac=0.1)
    W[3, 1] = np.inf
    W[40, 2] = np.nan
    W[77, 0] = -np.inf
    U = oracle_lib.prestack(F, A)
    for oob in (0, 1):
        bm, am = dropin_max(bplib, U, D, W, oob)
        obm, oam = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)
        beam = dropin_none(bplib, U, D, W, oob)
        ob = oracle_lib.beamform(U, D, W, oob)
        assert np.array_equal(bits(beam), bits(ob))


def test_nan_in_weighted_trace_propagates(cuda, bplib, oracle_lib):
    rng = np.random.default_rng(12)
    F, A, D, W = _random_problem(rng, 64, 4, 2, 600, 50, zero_frac=0.0)
    F[1, 0, 200:210] = np.nan
    U = oracle_lib.prestack(F, A)
    for oob in (0, 1):
        beam = dropin_none(bplib, U, D, W, oob)
        ob = oracle_lib.beamform(U, D, W, oob)
        assert np.array_equal(bits(beam), bits(ob))
        bm, am = dropin_max(bplib, U, D, W, oob)
        obm, oam = oracle_lib.beamform_max(U, D, W, oob)
        assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)


def test_minmax_kernel(cuda, bplib, oracle_lib):
    import torch
    from beampower_b200.tables import _stream_ptr
    rng = np.random.default_rng(3)
    _, _, D, W = _random_problem(rng, 1000, 7, 2, 10, 500, dmin=-200, zero_frac=0.5)
    W[17] = 0.0
    d = torch.from_numpy(D).cuda()
    w = torch.from_numpy(W).cuda()
    out = torch.empty((1000, 2), dtype=torch.int32, device="cuda")
    assert bplib.bp_minmax_dev(d.data_ptr(), w.data_ptr(), 1000, 7, 2, out.data_ptr(),
                               _stream_ptr()) == 0
    assert np.array_equal(out.cpu().numpy(), oracle_lib.minmax(D, W))


def test_direct_kernel_matches_staged(cuda, bplib):
    """Both GPU kernels agree bit for bit on one table."""
    import torch
    from beampower_b200.tables import TravelTimeTable, _stream_ptr
    rng = np.random.default_rng(9)
    F, A, D, W = _random_problem(rng, 300, 6, 2, 2000, 250)
    table = TravelTimeTable(D, W)
    tr = table.traces_from_features(F, A)
    for oob in (0, 1):
        bm, am = table.beamform_max(tr, oob)
        T = tr.n_samples
        keys = torch.empty(T, dtype=torch.int64, device="cuda")
        bm2 = torch.zeros(T, dtype=torch.float32, device="cuda")
        am2 = torch.zeros(T, dtype=torch.int32, device="cuda")
        rc = bplib.bp_beamform_max_direct_dev(tr.buf.data_ptr(), 0, None, T, tr.lpad, tr.pitch,
                                              table.delays.data_ptr(), table.weights.data_ptr(),
                                              300, 6, 2, oob, keys.data_ptr(), bm2.data_ptr(),
                                              am2.data_ptr(), _stream_ptr())
        assert rc == 0
        assert torch.equal(bm.view(torch.int32), bm2.view(torch.int32))
        assert torch.equal(am, am2)
    table.close()


def test_table_reuse_across_records(cuda, oracle_lib):
    """One resident table, several waveform records of different lengths."""
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(21)
    _, A, D, W = _random_problem(rng, 200, 5, 2, 10, 150)
    table = TravelTimeTable(D, W)
    for T in (100, 1000, 4097):
        F = np.abs(rng.standard_normal((5, 3, T))).astype(np.float32)
        tr = table.traces_from_features(F, A)
        U = oracle_lib.prestack(F, A)
        for oob in (0, 1):
            bm, am = table.beamform_max(tr, oob)
            obm, oam = oracle_lib.beamform_max(U, D, W, oob)
            assert np.array_equal(bits(bm.cpu().numpy()), bits(obm))
            assert np.array_equal(am.cpu().numpy(), oam)
    table.close()
