"""Every compiled shape of the staged kernel (sources per thread, samples per
lane, stations per ring stage, sources per block) gives the same results:
FP32 storage bit for bit against the oracle; 16-bit storage bit for bit
across shapes and against an exact model of its arithmetic.

The 16-bit model.  Traces are stored as U / scale_s rounded to the 16-bit
format (scale_s a power of two).  For a source whose station factors
c = w * scale_s are exact in that format (unit weights), the kernel adds
c * (phase sum) to an FP32 accumulator per station, stations ascending, with
one rounding per product: FP16 sums the phases in FP16 first, BF16 adds one
product per phase.  With w = 1 every product c * u is exact in FP32, so
NumPy's float32 `acc + c * u` reproduces each rounding.  Weights that are
not exact in the 16-bit format take the FP32-factor path, which gives the
same value per term; scaling every weight by 2^-30 moves FP16 factors below
its normal range (that path) and scales every beam by exactly 2^-30.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _configs(lib):
    return list(range(lib.bp_kernel_config_count()))


def _network(seed, S=10, C=3, P=2, N=300, T=5000, unit=True, spread=400):
    rng = np.random.default_rng(seed)
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, spread, size=(N, S, P)).astype(np.int32)
    if unit:
        W = np.ones((N, S), np.float32)
    else:
        W = rng.uniform(0.5, 1.5, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < 0.25] = 0.0
    return F, A, D, W


def _run(table, tr, oob, reduce):
    import torch
    if reduce == "max":
        bm, am = table.beamform_max(tr, oob)
        torch.cuda.synchronize()
        return bm.cpu().numpy(), am.cpu().numpy()
    beam = table.beamform(tr, oob)
    torch.cuda.synchronize()
    return beam.cpu().numpy()


def _with_config(lib, storage, reduce, cfg, fn):
    red = 1 if reduce == "max" else 0
    lib.bp_set_kernel_config(storage, red, cfg)
    try:
        return fn()
    finally:
        lib.bp_set_kernel_config(storage, red, -1)


def test_config_count_and_shapes(cuda, bplib):
    """At least six shapes, covering 8/16/32 samples per lane, 2/4/8 sources
    per thread and 1/2 stations per ring stage."""
    import ctypes as ct
    n = bplib.bp_kernel_config_count()
    assert n >= 6
    mts, kss, spss = set(), set(), set()
    for c in range(n):
        ks, mt, ws, ns = (ct.c_int() for _ in range(4))
        assert bplib.bp_kernel_config_describe(c, ct.byref(ks), ct.byref(mt), ct.byref(ws),
                                               ct.byref(ns)) == 0
        sps, kb, mb = (ct.c_int() for _ in range(3))
        assert bplib.bp_kernel_config_shape(c, ct.byref(sps), ct.byref(kb), ct.byref(mb)) == 0
        assert kb.value == ws.value * ks.value and 64 % kb.value == 0
        mts.add(mt.value)
        kss.add(ks.value)
        spss.add(sps.value)
    assert {8, 16, 32} <= mts and {2, 4, 8} <= kss and {1, 2} <= spss


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_every_shape_fp32_matches_oracle(cuda, bplib, oracle_lib, P):
    from beampower_b200.tables import TravelTimeTable
    F, A, D, W = _network(10 + P, P=P, unit=False)
    U = oracle_lib.prestack(F, A)
    ref = {oob: oracle_lib.beamform_max(U, D, W, oob) for oob in (0, 1)}
    ref_none = {oob: oracle_lib.beamform(U, D, W, oob) for oob in (0, 1)}
    table = TravelTimeTable(D, W)
    tr = table.traces_from_features(F, A, storage="fp32")
    for c in _configs(bplib):
        for oob in (0, 1):
            bm, am = _with_config(bplib, 0, "max", c, lambda: _run(table, tr, oob, "max"))
            assert np.array_equal(bm.view(np.uint32), ref[oob][0].view(np.uint32)), (c, oob)
            assert np.array_equal(am, ref[oob][1]), (c, oob)
            beam = _with_config(bplib, 0, "none", c, lambda: _run(table, tr, oob, "none"))
            assert np.array_equal(beam.view(np.uint32), ref_none[oob].view(np.uint32)), (c, oob)
    table.close()


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
@pytest.mark.parametrize("unit", [True, False])
def test_every_shape_16bit_identical(cuda, bplib, storage, unit):
    """The same 16-bit traces give the same bits in every shape, on the
    unit-weight (16-bit factor) path and on the FP32-factor path."""
    from beampower_b200.core import STORAGE
    from beampower_b200.tables import TravelTimeTable
    F, A, D, W = _network(21, unit=unit)
    table = TravelTimeTable(D, W)
    tr = table.traces_from_features(F, A, storage=storage)
    st = STORAGE[storage]
    for oob in (0, 1):
        outs = [_with_config(bplib, st, "max", c, lambda: _run(table, tr, oob, "max"))
                for c in _configs(bplib)]
        fulls = [_with_config(bplib, st, "none", c, lambda: _run(table, tr, oob, "none"))
                 for c in _configs(bplib)]
        for c in range(1, len(outs)):
            assert np.array_equal(outs[c][0].view(np.uint32), outs[0][0].view(np.uint32)), c
            assert np.array_equal(outs[c][1], outs[0][1]), c
            assert np.array_equal(fulls[c].view(np.uint32), fulls[0].view(np.uint32)), c
    table.close()


def _model_16bit(tr, D, W, storage, oob):
    """Exact float32 model of the 16-bit kernel for weights in {0, 1}."""
    from beampower_b200.core import trace_copies
    N, S, P = D.shape
    T = tr.n_samples
    rows = tr.buf[0::trace_copies(tr.storage)].float().cpu().numpy()  # (S * P, pitch)
    scales = tr.scales.cpu().numpy().astype(np.float32)
    pad = 3000
    V = np.zeros((S, P, T + 2 * pad), np.float32)
    V[:, :, pad:pad + T] = rows[:, tr.lpad:tr.lpad + T].reshape(S, P, T)
    t = np.arange(T)
    beam = np.zeros((N, T), np.float32)
    for i in range(N):
        acc = np.zeros(T, np.float32)
        ws = W[i] != 0
        if not ws.any():
            continue
        for s in range(S):
            if W[i, s] == 0:
                continue
            c = np.float32(W[i, s] * scales[s])
            u = [V[s, p, pad + t + D[i, s, p]] for p in range(P)]
            if storage == "fp16":
                ps = u[0].astype(np.float16)
                for p in range(1, P):
                    ps = (ps + u[p].astype(np.float16)).astype(np.float16)
                acc = (acc + c * ps.astype(np.float32)).astype(np.float32)
            else:
                for p in range(P):
                    acc = (acc + c * u[p]).astype(np.float32)
        if oob == 0:
            dmin = D[i][ws].min()
            dmax = D[i][ws].max()
            keep = (t + dmin >= 0) & (t + dmax < T)
            acc = np.where(keep, acc, np.float32(0))
        beam[i] = acc
    return beam


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_16bit_unit_weights_exact_model(cuda, bplib, storage, P):
    from beampower_b200.core import STORAGE
    from beampower_b200.tables import TravelTimeTable
    F, A, D, W = _network(30 + P, P=P, N=120, T=3000, unit=True)
    table = TravelTimeTable(D, W)
    tr = table.traces_from_features(F, A, storage=storage)
    st = STORAGE[storage]
    for oob in (0, 1):
        want = _model_16bit(tr, D, W, storage, oob)
        for c in _configs(bplib):
            beam = _with_config(bplib, st, "none", c, lambda: _run(table, tr, oob, "none"))
            assert np.array_equal(beam.view(np.uint32), want.view(np.uint32)), (c, oob)
    table.close()


def test_fp16_factor_paths_agree(cuda, bplib):
    """FP16: unit weights (16-bit factors) against weights 2^-30 (factors
    below FP16's normal range: the FP32-factor path) -- every beam scales by
    exactly 2^-30."""
    from beampower_b200.tables import TravelTimeTable
    F, A, D, W = _network(40, unit=True)
    tiny = np.float32(2.0 ** -30)
    t1 = TravelTimeTable(D, W)
    t2 = TravelTimeTable(D, W * tiny)
    tr1 = t1.traces_from_features(F, A, storage="fp16")
    tr2 = t2.traces_from_features(F, A, storage="fp16")
    assert np.array_equal(tr1.scales.cpu().numpy(), tr2.scales.cpu().numpy())
    for c in _configs(bplib):
        for oob in (0, 1):
            b1 = _with_config(bplib, 2, "none", c, lambda: _run(t1, tr1, oob, "none"))
            b2 = _with_config(bplib, 2, "none", c, lambda: _run(t2, tr2, oob, "none"))
            assert np.any(b1 != 0)
            assert np.array_equal((b2 / tiny).astype(np.float32).view(np.uint32),
                                  b1.view(np.uint32)), (c, oob)
    t1.close()
    t2.close()


def test_wide_windows_fall_back_correctly(cuda, bplib, oracle_lib):
    """Delay windows of ~2,600 samples: the 16-warp shapes keep a single
    atomic row for the cross-warp max (the per-warp rows would not leave room
    for the ring) and shapes that do not fit at all hand over to one that
    does; every choice stays bit for bit equal to the oracle."""
    from beampower_b200.tables import TravelTimeTable
    F, A, D, W = _network(50, S=6, N=300, T=6000, unit=False, spread=2600)
    U = oracle_lib.prestack(F, A)
    ref = oracle_lib.beamform_max(U, D, W, 0)
    table = TravelTimeTable(D, W)
    assert table.info["max_spread"] > 2000
    tr = table.traces_from_features(F, A, storage="fp32")
    used = set()
    for c in _configs(bplib):
        def run():
            used.add(bplib.bp_table_kernel_config(table.handle, 0, 1))
            return _run(table, tr, 0, "max")
        bm, am = _with_config(bplib, 0, "max", c, run)
        assert np.array_equal(bm.view(np.uint32), ref[0].view(np.uint32)), c
        assert np.array_equal(am, ref[1]), c
    assert {1, 2, 8} & used  # a 16-warp shape ran (with the single atomic row)
    table.close()


def _dequantized(tr, S, P):
    """(S, T, P) float32 traces from 16-bit rows: copy 0 times the station's
    (power-of-two) scale, exact."""
    from beampower_b200.core import trace_copies
    T = tr.n_samples
    rows = tr.buf[0::trace_copies(tr.storage)].float().cpu().numpy()[:, tr.lpad:tr.lpad + T]
    V = rows.reshape(S, P, T) * tr.scales.cpu().numpy().astype(np.float32)[:, None, None]
    return np.ascontiguousarray(V.astype(np.float32).transpose(0, 2, 1))


@pytest.mark.parametrize("unit", [True, False])
def test_windows_too_wide_for_16bit_rings(cuda, bplib, oracle_lib, unit):
    """Delay windows of ~4,500 samples: FP32 rings still fit a staged shape,
    the four 16-bit copies of every window fit none.  FP32 calls run the
    staged kernel; 16-bit calls expand their traces to FP32 (value times the
    power-of-two scale, exact) and run the same FP32 shapes, so both equal
    the oracle bit for bit -- the 16-bit ones on the dequantized traces."""
    from beampower_b200.tables import TravelTimeTable
    S, P = 6, 2
    F, A, D, W = _network(60, S=S, P=P, N=300, T=12000, unit=unit, spread=4500)
    table = TravelTimeTable(D, W)
    assert table.info["uses_window_kernel"] == 1
    assert table.info["max_spread"] > 4000
    assert bplib.bp_table_kernel_config(table.handle, 0, 1) >= 0
    for st in (1, 2):
        assert bplib.bp_table_kernel_config(table.handle, st, 1) == -1
        assert bplib.bp_table_kernel_config(table.handle, st, 0) == -1
    for storage in ("fp32", "fp16", "bf16"):
        tr = table.traces_from_features(F, A, storage=storage)
        U = oracle_lib.prestack(F, A) if storage == "fp32" else _dequantized(tr, S, P)
        for oob in (0, 1):
            ref_bm, ref_am = oracle_lib.beamform_max(U, D, W, oob)
            bm, am = _run(table, tr, oob, "max")
            assert np.array_equal(bm.view(np.uint32), ref_bm.view(np.uint32)), (storage, oob)
            assert np.array_equal(am, ref_am), (storage, oob)
            ref_full = oracle_lib.beamform(U, D, W, oob)
            beam = _run(table, tr, oob, "none")
            assert np.array_equal(beam.view(np.uint32), ref_full.view(np.uint32)), (storage, oob)
    table.close()


def test_stream_on_windows_too_wide_for_16bit_rings(cuda, bplib, oracle_lib):
    """A 16-bit stream on such a table stores FP32 instead and equals the
    oracle bit for bit; 16-bit records handed over directly are expanded to
    FP32 (the record path of the same fallback)."""
    import ctypes as ct
    import torch
    from beampower_b200.core import Record, STORAGE, check
    from beampower_b200.stream import NetworkStream
    from beampower_b200.tables import TravelTimeTable, _stream_ptr
    S, P = 6, 2
    F, A, D, W = _network(61, S=S, P=P, N=300, T=12000, unit=True, spread=4500)
    table = TravelTimeTable(D, W)
    U = oracle_lib.prestack(F, A)
    ref_bm, ref_am = oracle_lib.beamform_max(U, D, W, 0)
    ns = NetworkStream(table, A, storage="fp16")
    assert ns.storage == "fp32"
    for a in range(0, F.shape[2], 5000):
        ns.push(F[:, :, a:a + 5000])
    ns.flush()
    bm, am = ns.collect()
    assert np.array_equal(bm.view(np.uint32), ref_bm.view(np.uint32))
    assert np.array_equal(am, ref_am)
    # one 16-bit record over the whole trace, through the C-ABI
    tr = table.traces_from_features(F, A, storage="fp16")
    T = F.shape[2]
    bm16 = torch.zeros(T, dtype=torch.float32, device=tr.buf.device)
    am16 = torch.zeros(T, dtype=torch.int32, device=tr.buf.device)
    keys = torch.empty(T, dtype=torch.int64, device=tr.buf.device)
    r = Record()
    r.table, r.out_of_bounds = 0, 0
    r.traces, r.scales = tr.buf.data_ptr(), tr.scales.data_ptr()
    r.n_samples, r.lpad, r.pitch, r.t_origin, r.out0, r.out1 = T, tr.lpad, tr.pitch, 0, 0, T
    r.station_mask = None
    r.beam_max, r.argmax = bm16.data_ptr(), am16.data_ptr()
    check(bplib.bp_record_beamform_max_dev(table.handle, ct.byref(r), STORAGE["fp16"],
                                           keys.data_ptr(), _stream_ptr()))
    torch.cuda.synchronize()
    want_bm, want_am = oracle_lib.beamform_max(_dequantized(tr, S, P), D, W, 0)
    assert np.array_equal(bm16.cpu().numpy().view(np.uint32), want_bm.view(np.uint32))
    assert np.array_equal(am16.cpu().numpy(), want_am)
    table.close()


def test_batch_on_windows_too_wide_for_16bit_rings(cuda, oracle_lib):
    """A 16-bit batch that holds such a table stores FP32 traces instead
    (no 16-bit shape fits it) and gives the oracle's bits."""
    import torch
    from beampower_b200.batch import Window, WindowBatch
    from beampower_b200.tables import TravelTimeTable
    S, P = 6, 2
    F, A, D, W = _network(62, S=S, P=P, N=300, T=12000, unit=True, spread=4500)
    table = TravelTimeTable(D, W)
    batch = WindowBatch([table], [Window(0, F.shape[2])], A, storage="fp16")
    assert batch.storage == "fp32"
    batch.set_features(0, F)
    (bm, am), = batch.run()
    torch.cuda.synchronize()
    ref_bm, ref_am = oracle_lib.beamform_max(oracle_lib.prestack(F, A), D, W, 0)
    assert np.array_equal(bm.cpu().numpy().view(np.uint32), ref_bm.view(np.uint32))
    assert np.array_equal(am.cpu().numpy(), ref_am)
    batch.close()
    table.close()
