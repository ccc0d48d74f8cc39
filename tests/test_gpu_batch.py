"""Batch scheduler: windows of uneven length and station subset over two
resident tables, one persistent launch, CUDA-graph replay.  Every window's
result equals the oracle run on that window alone with the subset expressed
as zero weights (bit for bit with FP32 storage)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return np.where(np.isnan(a), np.uint32(0x7FC00000), a.view(np.uint32))


def _network(seed, S=12, C=3, P=2):
    rng = np.random.default_rng(seed)
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    grids = []
    for n, dmax in ((700, 260), (300, 90)):
        D = rng.integers(0, dmax + 1, size=(n, S, P)).astype(np.int32)
        W = rng.uniform(0.5, 1.5, size=(n, S)).astype(np.float32)
        W[rng.random(W.shape) < 0.15] = 0.0
        grids.append((D, W))
    return rng, A, grids


def _windows(rng, S):
    from beampower_b200.batch import Window
    specs = [(0, 5000, None, "strict"), (1, 777, [0, 3, 4, 9, 11], "strict"),
             (0, 1200, [1, 2, 5, 6, 7, 8], "flexible"), (1, 96, None, "flexible"),
             (0, 2600, list(range(0, S, 2)), "strict"), (1, 4100, [10], "strict")]
    return [Window(t, n, st, oob) for t, n, st, oob in specs]


def _expected(oracle_lib, A, grids, w, F):
    D, W = grids[w.table]
    if w.stations is not None:
        m = np.zeros(W.shape[1], dtype=np.float32)
        m[list(w.stations)] = 1.0
        W = W * m[None, :]
    U = oracle_lib.prestack(F, A)
    return oracle_lib.beamform_max(U, D, W, 0 if w.out_of_bounds == "strict" else 1)


@pytest.mark.parametrize("cfg", [-1, 0, 2, 3, 8])
def test_batch_matches_single_windows(cuda, oracle_lib, bplib, cfg):
    """Every window equals the oracle on that window alone, bit for bit, in
    the persistent kernel of the default shape and of shapes forced here."""
    import torch
    from beampower_b200.batch import WindowBatch
    from beampower_b200.tables import TravelTimeTable
    rng, A, grids = _network(1)
    tables = [TravelTimeTable(D, W) for D, W in grids]
    windows = _windows(rng, A.shape[0])
    bplib.bp_set_kernel_config(0, 1, cfg)
    try:
        batch = WindowBatch(tables, windows, A, storage="fp32")
    finally:
        bplib.bp_set_kernel_config(0, 1, -1)
    feats = []
    for i, w in enumerate(windows):
        F = np.abs(rng.standard_normal((A.shape[0], A.shape[1], w.n_samples))).astype(np.float32)
        feats.append(F)
        batch.set_features(i, F)
    out = batch.run()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for w, F, (bm, am) in zip(windows, feats, out):
        obm, oam = _expected(oracle_lib, A, grids, w, F)
        assert np.array_equal(bits(bm.cpu().numpy()), bits(obm)), w
        assert np.array_equal(am.cpu().numpy(), oam), w
    batch.close()
    for t in tables:
        t.close()


def test_batch_graph_replay_new_data(cuda, oracle_lib):
    """Capture once, replay on two further data sets in the same buffers."""
    import torch
    from beampower_b200.batch import WindowBatch
    from beampower_b200.tables import TravelTimeTable
    rng, A, grids = _network(2)
    tables = [TravelTimeTable(D, W) for D, W in grids]
    windows = _windows(rng, A.shape[0])
    batch = WindowBatch(tables, windows, A, storage="fp32")
    batch.capture()
    for _ in range(2):
        feats = []
        for i, w in enumerate(windows):
            F = np.abs(rng.standard_normal((A.shape[0], A.shape[1], w.n_samples))).astype(
                np.float32)
            feats.append(F)
            batch.set_features(i, F)
        out = batch.run()
        torch.cuda.synchronize()
        for w, F, (bm, am) in zip(windows, feats, out):
            obm, oam = _expected(oracle_lib, A, grids, w, F)
            assert np.array_equal(bits(bm.cpu().numpy()), bits(obm)), w
            assert np.array_equal(am.cpu().numpy(), oam), w
    batch.close()
    for t in tables:
        t.close()


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_batch_16bit_equals_single_window_16bit(cuda, storage):
    """16-bit batch results equal the single-window 16-bit path bit for bit
    (same per-(source, station) arithmetic; only the grouping differs)."""
    import torch
    import beampower_b200 as bp
    from beampower_b200.batch import WindowBatch
    from beampower_b200.tables import TravelTimeTable
    rng, A, grids = _network(3)
    tables = [TravelTimeTable(D, W) for D, W in grids]
    windows = _windows(rng, A.shape[0])
    batch = WindowBatch(tables, windows, A, storage=storage)
    feats = []
    for i, w in enumerate(windows):
        F = np.abs(rng.standard_normal((A.shape[0], A.shape[1], w.n_samples))).astype(np.float32)
        feats.append(F)
        batch.set_features(i, F)
    out = batch.run()
    torch.cuda.synchronize()
    for w, F, (bm, am) in zip(windows, feats, out):
        D, W = grids[w.table]
        if w.stations is not None:
            m = np.zeros(W.shape[1], dtype=np.float32)
            m[list(w.stations)] = 1.0
            W = W * m[None, :]
        ebm, eam = bp.beamform(F, D, A, W, reduce="max", out_of_bounds=w.out_of_bounds,
                               storage=storage)
        assert np.array_equal(bits(bm.cpu().numpy()), bits(ebm)), w
        assert np.array_equal(am.cpu().numpy(), eam), w
    batch.close()
