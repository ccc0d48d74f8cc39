"""16-bit trace storage (BF16 / FP16 with a power-of-two per-station scale,
FP32 accumulation) against the float64 restatement of the reference.

Tolerances, relative to |beam| in float64.  All terms of these cases have
one sign, so the beam's relative error is bounded by the relative roundings
each term goes through, plus FP32 accumulation (n 2^-24, below 1e-5 here):
  FP16 storage: 1e-3.  11 significant bits, unit roundoff 2^-11 = 4.9e-4;
    a term is rounded once when stored and once more in the FP16 sum of its
    phases: at most 2 x 4.9e-4 = 9.8e-4.
  BF16 storage: 4e-3.  8 significant bits, unit roundoff 2^-8 = 3.9e-3;
    a term is rounded once, when stored (each phase has its own FP32 FMA).
    BF16 therefore cannot promise 1e-3: a single stored value may be off by
    3.9e-3, and beams of few terms keep much of that (measured up to 2.9e-3
    on the small random cases, 1.7e-3 on the 4,000-source network).
Argmax: identical wherever the float64 top-two margin exceeds the tolerance.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

TOL = {"fp16": 1e-3, "bf16": 4e-3}


def _margin_mask(beam64, valid, tol):
    """Samples whose float64 winner beats the runner-up by more than tol."""
    b = np.where(valid, beam64, -np.inf)
    order = np.argsort(-b, axis=0)
    top1 = np.take_along_axis(b, order[:1], axis=0)[0]
    top2 = np.take_along_axis(b, order[1:2], axis=0)[0] if b.shape[0] > 1 else \
        np.full_like(top1, -np.inf)
    has = np.isfinite(top1)
    with np.errstate(invalid="ignore"):  # -inf - -inf where no source is valid
        margin = (top1 - top2) > tol * np.abs(top1)
    return has & margin, order[0], top1


def _check(orc, F, A, D, W, storage, oob, sources=None):
    import beampower_b200 as bp
    tol = TOL[storage]
    tag = "strict" if oob == 0 else "flexible"
    U64 = orc.fp64_prestack(F, A)
    beam64, valid = orc.fp64_beams(U64, D, W, oob)
    # full response
    beam = bp.beamform(F, D, A, W, reduce=None, out_of_bounds=tag, storage=storage)
    big = valid & (np.abs(beam64) > 1e-6 * np.abs(beam64).max())
    rel = np.abs(beam[big] - beam64[big]) / np.abs(beam64[big])
    assert rel.max() <= tol, (storage, tag, rel.max())
    assert np.all(beam[~valid] == 0)
    # max / argmax
    bm, am = bp.beamform(F, D, A, W, reduce="max", out_of_bounds=tag, storage=storage)
    sure, arg64, top1 = _margin_mask(beam64, valid, tol)
    assert np.array_equal(am[sure], arg64[sure]), (storage, tag)
    has = np.isfinite(top1)
    relm = np.abs(bm[has] - top1[has]) / np.maximum(np.abs(top1[has]), 1e-30)
    assert relm.max() <= tol, (storage, tag, relm.max())
    return rel.max(), relm.max()


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
@pytest.mark.parametrize("name", ["random_p2", "random_p1", "random_p3", "long_delays"])
def test_16bit_storage_within_tolerance(cuda, orc, storage, name):
    g = load_golden(name)
    for oob in (0, 1):
        _check(orc, g["F"], g["A"], g["D"], g["W"], storage, oob)


@pytest.mark.parametrize("spec_name", ["small-4k-src-20-sta-6000-samples", "small-heavy-tailed"])
def test_16bit_storage_small_network(cuda, orc, spec_name):
    """The 4,000-source network, Gaussian and heavy-tailed noise: the first
    1,000 sources against float64 (both storage types, strict)."""
    from beampower_b200.synthetic import SPECS, make_workload
    wl = make_workload(SPECS[spec_name])
    n = 1000
    F, A = wl["waveform_features"], wl["weights_phases"]
    D, W = wl["time_delays"][:n], wl["weights_sources"][:n]
    for storage in ("fp16", "bf16"):
        _check(orc, F, A, D, W, storage, 0)


def test_16bit_torch_path_and_scales(cuda, orc):
    """Device path: per-station scales are powers of two >= max |U|."""
    import torch
    from beampower_b200.tables import TravelTimeTable
    g = load_golden("random_p2")
    table = TravelTimeTable(g["D"], g["W"])
    for storage in ("fp16", "bf16"):
        tr = table.traces_from_features(g["F"], g["A"], storage=storage)
        sc = tr.scales.cpu().numpy()
        U = orc.fp64_prestack(g["F"], g["A"])
        mx = np.abs(U).max(axis=(1, 2))
        assert np.all(sc >= mx) and np.all(sc < 2 * mx + (mx == 0))
        assert np.all(np.log2(sc) == np.round(np.log2(sc)))
        back = tr.to_prestacked(g["U"].shape[2]).cpu().numpy()
        assert np.allclose(back, U, rtol=TOL[storage], atol=1e-6 * np.abs(U).max())
        bm, am = table.beamform_max(tr, 0)
        torch.cuda.synchronize()
    table.close()


def test_precision_report(cuda, orc, capsys):
    """Per-config error statement for 16-bit storage: the 4,000-source
    network with Gaussian and with heavy-tailed (Student-t, nu = 3) noise,
    all sources, strict rule; relative error of every computed beam and of
    beam_max against float64, and argmax agreement above the margin."""
    import json
    import beampower_b200 as bp
    from beampower_b200.synthetic import SMALL, SMALL_HEAVY, make_workload
    report = []
    for spec in (SMALL, SMALL_HEAVY):
        wl = make_workload(spec)
        F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                      wl["weights_sources"])
        beam64, valid = orc.fp64_beams(orc.fp64_prestack(F, A), D, W, 0)
        big = valid & (np.abs(beam64) > 1e-6 * np.abs(beam64).max())
        for storage in ("fp32", "fp16", "bf16"):
            tol = TOL.get(storage, 1e-5)
            beam = bp.beamform(F, D, A, W, reduce=None, storage=storage)
            rel = np.abs(beam[big] - beam64[big]) / np.abs(beam64[big])
            bm, am = bp.beamform(F, D, A, W, reduce="max", storage=storage)
            sure, arg64, top1 = _margin_mask(beam64, valid, tol)
            has = np.isfinite(top1)
            relm = np.abs(bm[has] - top1[has]) / np.abs(top1[has])
            row = {"config": spec.name, "storage": storage, "max_rel_beam": float(rel.max()),
                   "p999_rel_beam": float(np.percentile(rel, 99.9)),
                   "mean_rel_beam": float(rel.mean()), "max_rel_beam_max": float(relm.max()),
                   "argmax_above_margin_agree": float(np.mean(am[sure] == arg64[sure])),
                   "samples_above_margin": int(sure.sum()), "samples": int(has.sum())}
            report.append(row)
            assert row["max_rel_beam"] <= tol and row["argmax_above_margin_agree"] == 1.0
    with capsys.disabled():
        for row in report:
            print("PRECISION " + json.dumps(row))


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_16bit_nan_in_weighted_trace(cuda, orc, storage):
    """A NaN in a weighted station's trace: as in the FP32 path (and the
    reference), a NaN beam is never the maximum; samples whose every
    candidate beam is NaN keep 0 / argmax 0; the rest agree with float64
    within the storage tolerance, argmax identical above the margin."""
    import beampower_b200 as bp
    rng = np.random.default_rng(12)
    S, C, P, T, N = 4, 2, 2, 600, 64
    F = np.abs(rng.standard_normal((S, C, T))).astype(np.float32)
    A = rng.uniform(0.0, 1.5, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, 51, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.25, 2.0, size=(N, S)).astype(np.float32)
    F[1, 0, 200:210] = np.nan
    tol = TOL[storage]
    beam64, valid = orc.fp64_beams(orc.fp64_prestack(F, A), D, W, 0)
    finite = valid & np.isfinite(beam64)
    bm, am = bp.beamform(F, D, A, W, reduce="max", storage=storage)
    bm32, am32 = bp.beamform(F, D, A, W, reduce="max", storage="fp32")
    none = ~finite.any(axis=0)
    assert np.array_equal(bm[none], bm32[none]) and np.all(am[none] == 0) and none.any()
    b = np.where(finite, beam64, -np.inf)
    order = np.argsort(-b, axis=0)
    top1 = np.take_along_axis(b, order[:1], axis=0)[0]
    top2 = np.take_along_axis(b, order[1:2], axis=0)[0]
    has = ~none
    rel = np.abs(bm[has] - top1[has]) / np.abs(top1[has])
    assert rel.max() <= tol
    with np.errstate(invalid="ignore"):  # -inf - -inf at samples with no candidate
        sure = has & ((top1 - top2) > tol * np.abs(top1))
    assert np.array_equal(am[sure], order[0][sure])


@pytest.mark.parametrize("spec_name", ["small-4k-src-20-sta-6000-samples", "small-heavy-tailed"])
def test_scheduler_default_storage_within_1e3(cuda, orc, spec_name):
    """The batch and stream schedulers at their default storage (FP16):
    beam_max within 1e-3 of float64 and argmax identical above the margin,
    on the Gaussian and the heavy-tailed network (first 1,000 sources)."""
    import inspect
    import torch
    from beampower_b200.batch import Window, WindowBatch
    from beampower_b200.stream import NetworkStream
    from beampower_b200.synthetic import SPECS, make_workload
    from beampower_b200.tables import TravelTimeTable
    defaults = {inspect.signature(WindowBatch).parameters["storage"].default,
                inspect.signature(NetworkStream).parameters["storage"].default}
    assert defaults == {"fp16"}
    tol = 1e-3
    wl = make_workload(SPECS[spec_name])
    n = 1000
    F, A = wl["waveform_features"], wl["weights_phases"]
    D, W = wl["time_delays"][:n], wl["weights_sources"][:n]
    T = F.shape[2]
    beam64, valid = orc.fp64_beams(orc.fp64_prestack(F, A), D, W, 0)
    sure, arg64, top1 = _margin_mask(beam64, valid, tol)
    has = np.isfinite(top1)

    def check(bm, am, who):
        rel = np.abs(bm[has] - top1[has]) / np.abs(top1[has])
        assert rel.max() <= tol, (who, rel.max())
        assert np.array_equal(am[sure], arg64[sure]), who

    table = TravelTimeTable(D, W)
    batch = WindowBatch([table], [Window(0, T)], A)
    batch.set_features(0, F)
    (bm, am), = batch.run()
    torch.cuda.synchronize()
    check(bm.cpu().numpy(), am.cpu().numpy(), "batch")
    batch.close()
    ns = NetworkStream(table, A)
    for a in range(0, T, 1700):
        ns.push(F[:, :, a:a + 1700])
    ns.flush()
    bm, am = ns.collect()
    check(bm, am, "stream")
    table.close()
