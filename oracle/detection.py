"""CPU restatement of the tutorial's detection post-processing.

Test infrastructure: only the tests, ``smoke()`` and the benchmark's CPU legs
use this module, as the checker of the GPU detection path.

What it restates (file:line in the reference checkout):

* ``time_dependent_threshold`` -- notebooks/3_beampower.ipynb:497-579: zeros
  of the series are replaced by white noise scaled by the non-zero samples'
  centre and deviation; windows of ``sliding_window`` samples every
  ``int((1 - overlap) * sliding_window)`` samples give a centre and a
  deviation (mean/std for 'rms', median/median-absolute-deviation for 'mad');
  ``centre + num_dev * deviation`` is max-filtered with both neighbours and
  spread back to every sample.  The white noise is an argument here (the
  notebook draws it from NumPy's global generator), so that results can be
  compared.
* the detection cell -- notebooks/3_beampower.ipynb:618-626:
  ``scipy.signal.find_peaks(beam_max, distance=...)`` then the peaks whose
  height is strictly above the threshold.

SciPy (1.18.1 in this image) is a third-party dependency of the tutorial.  Its
peak finder is restated here from its published algorithm
(scipy/signal/_peak_finding_utils.pyx: ``_local_maxima_1d``,
``_select_by_peak_distance``, ``_peak_prominences``; scipy/signal/
_peak_finding.py: the height / threshold / prominence conditions), and the
tests compare this restatement with SciPy itself.  The tutorial uses
``distance`` and shows ``prominence`` with ``wlen`` as an option
(notebooks/3_beampower.ipynb:625).  Where SciPy orders equal peak heights
through NumPy's (unstable) default argsort, this restatement uses the stable
order: among equal heights the later sample is considered first.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def time_dependent_threshold(time_series, sliding_window, overlap=0.66, threshold_type="rms",
                             num_dev=8.0, white_noise=None):
    """Threshold of the same length as ``time_series`` (float32).

    white_noise: standard normal draws, one per zero sample in series order
    (the notebook's ``np.random.normal(size=n_zeros).astype("float32")``).
    """
    ts = np.array(time_series, dtype=F32, copy=True)
    kind = threshold_type.lower()
    n = ts.shape[0]
    W = int(sliding_window)
    half = W // 2
    shift = int((1.0 - overlap) * W)
    if W < 1 or n <= W:
        raise ValueError("the series must be longer than the sliding window")
    if shift < 1:
        raise ValueError("(1 - overlap) * sliding_window must be at least 1")
    zeros = ts == 0.0
    n_zeros = int(zeros.sum())
    noise = np.zeros(0, F32) if white_noise is None else np.asarray(white_noise, F32)
    if noise.shape[0] < n_zeros:
        raise ValueError(f"white_noise holds {noise.shape[0]} values, {n_zeros} zeros")
    nz = ts[~zeros]
    with np.errstate(invalid="ignore", divide="ignore"):
        if kind == "rms":
            centre0 = nz.mean() if nz.size else F32(np.nan)
            dev0 = np.std(nz) if nz.size else F32(np.nan)
        elif kind == "mad":
            centre0 = np.median(nz) if nz.size else F32(np.nan)
            dev0 = np.median(np.abs(nz - centre0)) if nz.size else F32(np.nan)
        else:
            raise ValueError("threshold_type must be 'rms' or 'mad'")
    ts[zeros] = noise[:n_zeros] * F32(dev0) + F32(centre0)
    win = np.lib.stride_tricks.sliding_window_view(ts, W)[::shift, :]
    if kind == "rms":
        centre = np.mean(win, axis=-1)
        dev = np.std(win, axis=-1)
    else:
        centre = np.median(win, axis=-1)
        dev = np.median(np.abs(win - centre[:, None]), axis=-1)
    thr = (centre + F32(num_dev) * dev).astype(F32)
    t1 = thr.copy()
    t1[1:] = np.maximum(thr[:-1], thr[1:])
    t2 = t1.copy()
    t2[:-1] = np.maximum(t1[:-1], t1[1:])
    idx = np.arange(half, n - (W - half)) // shift
    idx[idx >= t2.shape[0]] = t2.shape[0] - 1
    mid = t2[idx]
    return np.concatenate([np.full(half, mid[0], F32), mid,
                           np.full(W - half, mid[-1], F32)]).astype(F32)


def local_maxima(x):
    """(left edges, right edges, midpoints) of every local maximum, flat
    plateaus included (a plateau counts when its both neighbours are lower)."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[0]
    mids, lefts, rights = [], [], []
    i, i_max = 1, n - 1
    while i < i_max:
        if x[i - 1] < x[i]:
            j = i + 1
            while j < i_max and x[j] == x[i]:
                j += 1
            if x[j] < x[i]:
                lefts.append(i)
                rights.append(j - 1)
                mids.append((i + j - 1) // 2)
                i = j
        i += 1
    return (np.array(lefts, np.int64), np.array(rights, np.int64), np.array(mids, np.int64))


def select_by_distance(peaks, priority, distance):
    """Keep-mask: peaks in decreasing priority keep themselves and drop every
    other peak closer than ``ceil(distance)`` samples."""
    peaks = np.asarray(peaks, np.int64)
    m = peaks.shape[0]
    d = math.ceil(distance)
    keep = np.ones(m, dtype=bool)
    order = np.argsort(np.asarray(priority), kind="stable")
    for i in range(m - 1, -1, -1):
        j = order[i]
        if not keep[j]:
            continue
        k = j - 1
        while k >= 0 and peaks[j] - peaks[k] < d:
            keep[k] = False
            k -= 1
        k = j + 1
        while k < m and peaks[k] - peaks[j] < d:
            keep[k] = False
            k += 1
    return keep


def interval_borders(interval, x, peaks):
    """(min, max) borders of a height / prominence condition: a number, a
    pair, or arrays over x read at the peaks (SciPy's condition arguments)."""
    try:
        lo, hi = interval
    except (TypeError, ValueError):
        lo, hi = interval, None
    if isinstance(lo, np.ndarray):
        if lo.size != x.size:
            raise ValueError("array size of lower interval border must match x")
        lo = lo[peaks]
    if isinstance(hi, np.ndarray):
        if hi.size != x.size:
            raise ValueError("array size of upper interval border must match x")
        hi = hi[peaks]
    return lo, hi


def within(values, lo, hi):
    keep = np.ones(values.size, dtype=bool)
    if lo is not None:
        keep &= lo <= values
    if hi is not None:
        keep &= values <= hi
    return keep


def peak_prominences(x, peaks, wlen=None):
    """(prominences, left_bases, right_bases): from each peak, walk outwards
    while the signal is not above the peak (at most wlen // 2 samples when
    wlen is given); the base on each side is the lowest sample met, the
    prominence the peak minus the higher of the two bases (float64)."""
    x = np.asarray(x, np.float64)
    w = -1 if wlen is None else math.ceil(wlen)
    if wlen is not None and w <= 1:
        raise ValueError(f"`wlen` must be larger than 1, was {w}")
    n = x.shape[0]
    prom = np.empty(len(peaks), np.float64)
    lb = np.empty(len(peaks), np.int64)
    rb = np.empty(len(peaks), np.int64)
    for k, pk in enumerate(peaks):
        lo_end, hi_end = 0, n - 1
        if w >= 2:
            lo_end = max(pk - w // 2, lo_end)
            hi_end = min(pk + w // 2, hi_end)
        i = lb[k] = pk
        left = x[pk]
        while lo_end <= i and x[i] <= x[pk]:
            if x[i] < left:
                left = x[i]
                lb[k] = i
            i -= 1
        i = rb[k] = pk
        right = x[pk]
        while i <= hi_end and x[i] <= x[pk]:
            if x[i] < right:
                right = x[i]
                rb[k] = i
            i += 1
        prom[k] = x[pk] - max(left, right)
    return prom, lb, rb


def find_peaks(x, distance=None, height=None, prominence=None, wlen=None, properties=False,
               threshold=None):
    """Peaks of x as scipy.signal.find_peaks(x, height=, threshold=,
    distance=, prominence=, wlen=): local maxima, then the height condition,
    the threshold condition, the distance rule and the prominence condition,
    in SciPy's order.  Returns the indexes, or (indexes, properties) with
    ``properties=True``."""
    x = np.asarray(x)
    if x.ndim != 1:
        raise ValueError("x must be one-dimensional")
    x64 = np.asarray(x, np.float64)
    _l, _r, peaks = local_maxima(x)
    props = {}
    if height is not None:
        h = x64[peaks]
        lo, hi = interval_borders(height, x64, peaks)
        keep = within(h, lo, hi)
        peaks = peaks[keep]
        props["peak_heights"] = h[keep]
    if threshold is not None:
        # the rise over each neighbour; the smaller one against the lower
        # border, the larger one against the upper border
        left = x64[peaks] - x64[peaks - 1]
        right = x64[peaks] - x64[peaks + 1]
        lo, hi = interval_borders(threshold, x64, peaks)
        keep = np.ones(peaks.size, dtype=bool)
        if lo is not None:
            keep &= lo <= np.minimum(left, right)
        if hi is not None:
            keep &= np.maximum(left, right) <= hi
        peaks = peaks[keep]
        props = {k: v[keep] for k, v in props.items()}
        props.update(left_thresholds=left[keep], right_thresholds=right[keep])
    if distance is not None:
        if distance < 1:
            raise ValueError("distance must be greater or equal to 1")
        keep = select_by_distance(peaks, x64[peaks], distance)
        peaks = peaks[keep]
        props = {k: v[keep] for k, v in props.items()}
    if prominence is not None:
        prom, lb, rb = peak_prominences(x64, peaks, wlen)
        props.update(prominences=prom, left_bases=lb, right_bases=rb)
        lo, hi = interval_borders(prominence, x64, peaks)
        keep = within(prom, lo, hi)
        peaks = peaks[keep]
        props = {k: v[keep] for k, v in props.items()}
    return (peaks, props) if properties else peaks


def detect(beam_max, threshold, distance):
    """Detections of the tutorial: peaks of beam_max at least ``distance``
    samples apart whose height is strictly above the threshold."""
    bm = np.asarray(beam_max, F32)
    peaks = find_peaks(bm, distance=distance)
    return peaks[bm[peaks] > np.asarray(threshold, F32)[peaks]]
