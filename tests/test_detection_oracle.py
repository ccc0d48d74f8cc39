"""CPU checks of the detection step's oracle and of the summation order the
GPU threshold reproduces.

* The oracle (oracle/detection.py) against the golden fixtures made from
  the reference tutorial's own ``time_dependent_threshold`` and SciPy's
  ``find_peaks`` (tests/golden/make_detection_golden.py): bit for bit.
* The oracle's peak finder against SciPy itself on seeded series.
* ``bp_pairwise_sum_f32`` (the library's host evaluation of the split tree
  its threshold kernels use) against NumPy's float32 sum, bit for bit.
"""
import glob
import os

import numpy as np
import pytest
from scipy import signal

from conftest import GOLDEN

from oracle import detection as odet

CASES = sorted(os.path.basename(p)[len("detection_"):-len(".npz")]
               for p in glob.glob(os.path.join(GOLDEN, "detection_*.npz")))


def load_detection(name):
    with np.load(os.path.join(GOLDEN, f"detection_{name}.npz")) as z:
        g = {k: z[k] for k in z.files}
    g["distance"] = None if float(g["distance"]) < 0 else float(g["distance"])
    return g


def bits(a):
    a = np.asarray(a, np.float32).copy()
    a[np.isnan(a)] = np.float32(np.nan)
    return a.view(np.uint32)


def test_fixtures_present():
    assert len(CASES) >= 8


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_tutorial_fixtures(name):
    g = load_detection(name)
    thr = odet.time_dependent_threshold(g["x"], int(g["window"]), float(g["overlap"]),
                                        str(g["kind"]), float(g["num_dev"]), g["noise"])
    assert np.array_equal(bits(thr), bits(g["threshold"]))
    assert np.array_equal(odet.find_peaks(g["x"], g["distance"]), g["peaks"])
    assert np.array_equal(odet.detect(g["x"], thr, g["distance"]), g["detections"])


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("distance", [None, 1, 2.5, 17, 400])
def test_oracle_peaks_match_scipy(seed, distance):
    rng = np.random.default_rng(seed)
    x = np.convolve(rng.standard_normal(5000), np.ones(7) / 7, mode="same").astype(np.float32)
    x[1000:1010] = x[1000]  # a plateau
    x[3000:3500] = 0.0      # a zero run
    ref = signal.find_peaks(x, distance=distance)[0]
    assert np.array_equal(odet.find_peaks(x, distance), ref)


def test_oracle_edge_cases():
    with pytest.raises(ValueError):
        odet.time_dependent_threshold(np.ones(100, np.float32), 100)
    with pytest.raises(ValueError):
        odet.time_dependent_threshold(np.ones(100, np.float32), 10, overlap=0.99)
    with pytest.raises(ValueError):
        odet.find_peaks(np.ones(10, np.float32), 0.5)
    assert odet.find_peaks(np.array([1.0, 2.0], np.float32)).size == 0
    # equal heights closer than the distance: the later one is kept
    x = np.zeros(50, np.float32)
    x[10] = x[14] = 3.0
    assert list(odet.find_peaks(x, 10)) == [14]


def test_pairwise_sum_tree_matches_numpy(bplib):
    import ctypes as ct
    rng = np.random.default_rng(7)
    sizes = list(range(0, 300)) + [1023, 1024, 1025, 4097, 65537, 180000, 180001, 999983]
    for n in sizes:
        a = (rng.standard_normal(n) * rng.uniform(0.1, 1e4)).astype(np.float32)
        got = bplib.bp_pairwise_sum_f32(a.ctypes.data_as(ct.c_void_p), n)
        want = np.sum(a)
        assert np.float32(got).view(np.uint32) == np.float32(want).view(np.uint32), n


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("kw", [
    {"height": 0.2}, {"height": (0.1, 0.6)}, {"height": "array"},
    {"prominence": 0.3}, {"prominence": (0.2, 1.5), "wlen": 25},
    {"prominence": 0.1, "wlen": 7.5}, {"height": 0.0, "distance": 40, "prominence": 0.25},
    {"distance": 12, "prominence": (None, 0.8), "wlen": 100},
    {"threshold": 0.02}, {"threshold": (0.01, 0.2)}, {"threshold": (None, 0.05)},
    {"threshold": "array", "distance": 8}, {"height": 0.1, "threshold": 0.01, "prominence": 0.2},
    {"prominence": "array", "wlen": 60}, {"prominence": ("array", 2.0)}])
def test_oracle_peak_options_match_scipy(seed, kw):
    rng = np.random.default_rng(seed)
    x = np.convolve(rng.standard_normal(4000), np.ones(5) / 5, mode="same").astype(np.float32)
    x[700:706] = x[700]
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
    ref, ref_props = signal.find_peaks(x, **kw)
    got, props = odet.find_peaks(x, properties=True, **kw)
    assert np.array_equal(got, ref)
    assert set(props) == set(ref_props)
    for k in props:
        assert np.array_equal(props[k], ref_props[k]), k
