"""The autotuner times every kernel shape, keeps the fastest, and every shape
gives the same results (FP32: bit for bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_selects_and_results_agree(cuda, tmp_path, monkeypatch):
    import torch
    from beampower_b200 import autotune
    from beampower_b200.core import load_library
    from beampower_b200.tables import TravelTimeTable
    monkeypatch.setenv(autotune.CACHE_ENV, str(tmp_path / "cache.json"))
    lib = load_library("gpu")
    rng = np.random.default_rng(4)
    S, C, P, N, T = 9, 3, 2, 900, 7000
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, 300, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.5, 1.5, size=(N, S)).astype(np.float32)
    table = TravelTimeTable(D, W)
    for storage in ("fp32", "fp16"):
        tr = table.traces_from_features(F, A, storage=storage)
        res = autotune.autotune(table, tr, repeats=1)
        assert set(res["times_ms"]) == {c for c, _ in autotune.configs()}
        ran = {c: t for c, t in res["times_ms"].items() if t is not None}
        assert res["best"] == min(ran, key=ran.get)
        for c in res["times_ms"]:  # every shape fits this small table
            assert lib.bp_table_kernel_config(table.handle, tr.storage, 1) in range(
                lib.bp_kernel_config_count())
            assert res["times_ms"][c] is not None
        outs = []
        for c, _ in autotune.configs():
            lib.bp_set_kernel_config(tr.storage, 1, c)
            bm, am = table.beamform_max(tr, 0)
            torch.cuda.synchronize()
            outs.append((bm.cpu().numpy().view(np.uint32), am.cpu().numpy()))
        for o in outs[1:]:
            assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])
        lib.bp_set_kernel_config(tr.storage, 1, -1)
        assert autotune.apply_cached(table, storage) == res["best"]
        lib.bp_set_kernel_config(tr.storage, 1, -1)
    table.close()
