"""Detection on the GPU against the tutorial fixtures and the oracle.

Everything here is exact: the threshold bit for bit (float32 in NumPy's
order), peak and detection indexes equal.
* golden fixtures made from the reference tutorial's own function and SciPy;
* a day-long series (2,160,000 samples: 24 h at 25 Hz) with the tutorial's
  settings (7,200 s windows, 60 s minimum distance), against the oracle;
* the C2-size beam series shape (180,000 samples) with both threshold rules;
* the library's own noise for zero samples, edge cases and errors.
"""
import numpy as np
import pytest

from test_detection_oracle import CASES, bits, load_detection

pytestmark = pytest.mark.gpu


def _det():
    import beampower_b200.detection as det
    return det


@pytest.mark.parametrize("name", CASES)
def test_threshold_matches_tutorial_fixtures(cuda, name):
    g = load_detection(name)
    thr = _det().time_dependent_threshold(g["x"], int(g["window"]), float(g["overlap"]),
                                          str(g["kind"]), float(g["num_dev"]),
                                          white_noise=g["noise"])
    assert np.array_equal(bits(thr), bits(g["threshold"]))


@pytest.mark.parametrize("name", CASES)
def test_peaks_and_detections_match_tutorial_fixtures(cuda, name):
    g = load_detection(name)
    peaks, props = _det().find_peaks(g["x"], distance=g["distance"])
    assert props == {}
    assert peaks.dtype == np.int64 and np.array_equal(peaks, g["peaks"])
    argmax = (np.arange(g["x"].size) * 7 % 1000).astype(np.int32)
    d = _det().detect(g["x"], argmax, threshold=g["threshold"], distance=g["distance"])
    assert np.array_equal(d.peaks, g["detections"])
    assert np.array_equal(bits(d.heights), bits(g["x"][g["detections"]]))
    assert np.array_equal(d.sources, argmax[g["detections"]])


def _day_series(seed, n, zero_tail):
    rng = np.random.default_rng(seed)
    x = np.abs(rng.standard_normal(n + 24)).astype(np.float32)
    x = np.convolve(x, np.ones(25, np.float32) / 25, mode="valid")[:n].astype(np.float32) * 10
    t0 = rng.integers(1000, n - zero_tail - 1000, size=200)
    for t in t0:
        lo, hi = max(t - 40, 0), min(t + 40, n)
        x[lo:hi] += (rng.uniform(5, 30) * np.exp(-0.5 * ((np.arange(lo, hi) - t) / 6.0) ** 2)
                     ).astype(np.float32)
    x[n - zero_tail:] = 0.0
    return x


@pytest.mark.parametrize("kind", ["rms", "mad"])
def test_day_long_series_against_oracle(cuda, kind):
    from oracle import detection as odet
    fs = 25.0
    n = int(24 * 3600 * fs)
    x = _day_series(11, n, 2864)
    W, dist = int(7200.0 * fs), int(60 * fs)
    noise = np.random.default_rng(5).standard_normal(int((x == 0).sum())).astype(np.float32)
    thr = _det().time_dependent_threshold(x, W, 0.66, kind, 8.0, white_noise=noise)
    ref = odet.time_dependent_threshold(x, W, 0.66, kind, 8.0, noise)
    assert np.array_equal(bits(thr), bits(ref))
    peaks, _ = _det().find_peaks(x, distance=dist)
    assert np.array_equal(peaks, odet.find_peaks(x, dist))
    d = _det().detect(x, threshold=thr, distance=dist)
    assert np.array_equal(d.peaks, odet.detect(x, ref, dist))


@pytest.mark.parametrize("kind,num_dev", [("rms", 3.0), ("mad", 6.0)])
def test_beam_series_180k_against_oracle(cuda, kind, num_dev):
    import torch
    from oracle import detection as odet
    x = _day_series(12, 180000, 2864)
    x[:100] = 0.0
    noise = np.random.default_rng(6).standard_normal(int((x == 0).sum())).astype(np.float32)
    xt = torch.from_numpy(x).to(cuda)
    thr = _det().time_dependent_threshold(xt, 20000, 0.66, kind, num_dev,
                                          white_noise=torch.from_numpy(noise).to(cuda))
    assert isinstance(thr, torch.Tensor) and thr.is_cuda
    ref = odet.time_dependent_threshold(x, 20000, 0.66, kind, num_dev, noise)
    assert np.array_equal(bits(thr.cpu().numpy()), bits(ref))
    d = _det().detect(xt, threshold=thr, distance=250)
    assert np.array_equal(d.peaks.cpu().numpy(), odet.detect(x, ref, 250))


def test_generated_noise_is_seeded(cuda):
    from oracle import detection as odet
    x = _day_series(13, 30000, 3000)
    a = _det().time_dependent_threshold(x, 4000, seed=1)
    b = _det().time_dependent_threshold(x, 4000, seed=1)
    c = _det().time_dependent_threshold(x, 4000, seed=2)
    assert np.array_equal(bits(a), bits(b)) and np.isfinite(a).all()
    assert not np.array_equal(a, c)
    # without zero samples the noise plays no part: equal to the oracle
    y = x[:25000].copy()
    assert (y != 0).all()
    assert np.array_equal(bits(_det().time_dependent_threshold(y, 4000, seed=3)),
                          bits(odet.time_dependent_threshold(y, 4000)))


def test_edge_cases(cuda):
    from oracle import detection as odet
    det = _det()
    with pytest.raises(ValueError):
        det.time_dependent_threshold(np.ones(100, np.float32), 100)
    with pytest.raises(ValueError):
        det.time_dependent_threshold(np.ones(100, np.float32), 10, overlap=0.99)
    with pytest.raises(ValueError):
        det.find_peaks(np.ones(10, np.float32), distance=0.5)
    for n in (0, 1, 2):
        assert det.find_peaks(np.zeros(n, np.float32))[0].size == 0
    # a series of zeros: NaN threshold, as NumPy's mean of nothing
    z = det.time_dependent_threshold(np.zeros(500, np.float32), 100,
                                     white_noise=np.ones(500, np.float32))
    assert np.isnan(z).all()
    # equal heights within the distance, plateaus, NaN and infinities
    x = np.zeros(200, np.float32)
    x[10] = x[14] = 3.0
    x[50:55] = 2.0
    x[80] = np.nan
    x[100] = np.inf
    x[120], x[121] = 5.0, 5.0
    for dist in (None, 1, 3, 10, 45):
        assert np.array_equal(det.find_peaks(x, distance=dist)[0], odet.find_peaks(x, dist))


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("kw", [
    {"height": 0.2}, {"height": (0.1, 0.6)}, {"height": "array"},
    {"prominence": 0.3}, {"prominence": (0.2, 1.5), "wlen": 25},
    {"prominence": 0.1, "wlen": 7.5}, {"height": 0.0, "distance": 40, "prominence": 0.25},
    {"distance": 12, "prominence": (None, 0.8), "wlen": 100},
    {"threshold": 0.02}, {"threshold": (0.01, 0.2)}, {"threshold": (None, 0.05)},
    {"threshold": "array", "distance": 8}, {"height": 0.1, "threshold": 0.01, "prominence": 0.2},
    {"prominence": "array", "wlen": 60}, {"prominence": ("array", 2.0)}])
def test_peak_options_match_oracle(cuda, seed, kw):
    """height / prominence / wlen (the tutorial's commented option at
    notebooks/3_beampower.ipynb:625): identical peaks and properties."""
    from oracle import detection as odet
    rng = np.random.default_rng(seed)
    x = np.convolve(rng.standard_normal(40000), np.ones(5) / 5, mode="same").astype(np.float32)
    x[700:706] = x[700]
    x[9000:9400] = 0.0
    kw = dict(kw)
    wave = 0.1 + 0.2 * np.sin(np.arange(x.size) / 300.0)
    if kw.get("height") == "array":
        kw["height"] = wave.astype(np.float32)
    if kw.get("threshold") == "array":
        kw["threshold"] = 0.1 * wave  # float64 borders, compared in float64
    if kw.get("prominence") == "array":
        kw["prominence"] = 2.0 * wave
    if isinstance(kw.get("prominence"), tuple) and kw["prominence"][0] == "array":
        kw["prominence"] = (wave, kw["prominence"][1])
    ref, ref_props = odet.find_peaks(x, properties=True, **kw)
    got, props = _det().find_peaks(x, **kw)
    assert np.array_equal(got, ref)
    assert set(props) == set(ref_props)
    for k in props:
        assert np.array_equal(props[k], ref_props[k]), k


def test_prominence_without_window_on_a_day(cuda):
    """Prominence walks with no window over a day-long series (the highest
    peaks walk to the series ends), against SciPy itself (the oracle's walk
    in Python would take minutes here; it is checked against SciPy on the
    CPU)."""
    from scipy import signal
    x = _day_series(14, 2_160_000, 2864)
    ref, ref_props = signal.find_peaks(x, distance=1500, prominence=20.0)
    got, props = _det().find_peaks(x, distance=1500, prominence=20.0)
    assert ref.size > 10 and np.array_equal(got, ref)
    for k in ("prominences", "left_bases", "right_bases"):
        assert np.array_equal(props[k], ref_props[k]), k
