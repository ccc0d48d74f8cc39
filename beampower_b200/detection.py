"""Detection on the beam series, on the GPU.

The reference tutorial turns ``beam_max`` into detections in two notebook
cells: a time-dependent threshold (notebooks/3_beampower.ipynb:497-579,
``time_dependent_threshold``) and ``scipy.signal.find_peaks(beam_max,
distance=...)`` followed by the strict threshold test
(notebooks/3_beampower.ipynb:618-626).  The functions here run both on the
device and give identical results: float32 arithmetic in NumPy's order for
the threshold, SciPy's rules for the peaks.

Inputs are numpy arrays or torch tensors; CUDA tensors stay on their device.
Outputs follow the input: numpy in, numpy out; tensor in, tensor out.
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass

import numpy as np

from .core import PeakOptions, check, load_library

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None

THRESHOLD_KINDS = {"rms": 0, "mad": 1}


def _as_device(x, dtype):
    from .tables import _dev_tensor
    if torch is None:
        raise RuntimeError("torch is required for the detection functions")
    dev = x.device if isinstance(x, torch.Tensor) and x.is_cuda else torch.device(
        "cuda", torch.cuda.current_device())
    return _dev_tensor(x, dtype, dev)


def _is_tensor(x):
    return torch is not None and isinstance(x, torch.Tensor)


def _out(t, like):
    return t if _is_tensor(like) else t.cpu().numpy()


def time_dependent_threshold(time_series, sliding_window, overlap=0.66, threshold_type="rms",
                             num_dev=8.0, white_noise=None, seed=0):
    """Per-sample detection threshold of a beam series (float32).

    Same arguments and result as the tutorial's ``time_dependent_threshold``
    (notebooks/3_beampower.ipynb:497): zero samples are replaced by white
    noise scaled by the non-zero samples' centre and deviation; every
    ``int((1 - overlap) * sliding_window)`` samples a window of
    ``sliding_window`` samples gives centre + num_dev * deviation (mean and
    standard deviation for 'rms', median and median absolute deviation for
    'mad'); the window values are max-filtered with their neighbours and
    spread back to every sample.

    white_noise: the standard normal draws for the zero samples, in sample
    order (the tutorial draws ``np.random.normal(size=n_zeros)``); when None
    they come from this library's generator seeded by ``seed``.
    """
    lib = load_library("gpu")
    kind = THRESHOLD_KINDS.get(str(threshold_type).lower())
    if kind is None:
        raise ValueError("threshold_type must be 'rms' or 'mad'")
    x = _as_device(time_series, torch.float32)
    if x.ndim != 1:
        raise ValueError("time_series must be one-dimensional")
    n = int(x.shape[0])
    out = torch.empty(n, dtype=torch.float32, device=x.device)
    noise_ptr, n_noise = None, 0
    if white_noise is not None:
        noise = _as_device(white_noise, torch.float32).reshape(-1)
        noise_ptr, n_noise = noise.data_ptr(), int(noise.shape[0])
    from .tables import _stream_ptr
    with torch.cuda.device(x.device):
        rc = lib.bp_threshold_dev(x.data_ptr(), n, int(sliding_window), float(overlap), kind,
                                  float(num_dev), noise_ptr, n_noise, int(seed) & (2**64 - 1),
                                  out.data_ptr(), _stream_ptr())
    if rc == 1:
        raise ValueError(lib.bp_last_error().decode())
    check(rc)
    return _out(out, time_series)


def _borders(interval, n, device):
    """SciPy's condition argument -> (min, max, min array, max array): a
    number, a pair, or arrays over the series (read at the peaks)."""
    try:
        lo, hi = interval
    except (TypeError, ValueError):
        lo, hi = interval, None

    def one(v):
        if v is None:
            return float("nan"), None
        if isinstance(v, np.ndarray) or _is_tensor(v):
            a = _as_device(v, torch.float64).reshape(-1)
            if a.numel() != n:
                raise ValueError("array size of interval border must match x")
            return float("nan"), a
        return float(v), None

    (lo_v, lo_a), (hi_v, hi_a) = one(lo), one(hi)
    return lo_v, hi_v, lo_a, hi_a


def find_peaks(x, height=None, threshold=None, distance=None, prominence=None, width=None,
               wlen=None, rel_height=0.5, plateau_size=None):
    """``(peaks, properties)`` as ``scipy.signal.find_peaks(x, height=,
    threshold=, distance=, prominence=, wlen=)``, with SciPy's parameter
    order; ``width`` and ``plateau_size`` are not implemented and raise
    NotImplementedError when given.

    Peaks are the local maxima of x (a flat plateau counts at its midpoint
    when both its neighbours are lower), then, in SciPy's order: the height
    condition, the threshold condition (the peak's rise over each neighbour:
    the smaller rise against the lower border, the larger against the upper),
    the minimum distance (peaks taken in decreasing height; every peak closer
    than ``ceil(distance)`` samples to a taken one is dropped; equal heights:
    the later sample first, where SciPy leaves the order to NumPy's unstable
    sort), and the prominence condition (walks limited to ``wlen``).  Each
    condition takes a number, a (min, max) pair with None for an open side,
    or per-sample arrays read at the peaks, as SciPy does.
    properties: ``peak_heights`` with height; ``left_thresholds``,
    ``right_thresholds`` with threshold; ``prominences``, ``left_bases``,
    ``right_bases`` with prominence, as SciPy returns them (float64 values,
    int64 indexes).
    """
    for name, v in (("width", width), ("plateau_size", plateau_size)):
        if v is not None:
            raise NotImplementedError(f"find_peaks: `{name}` is not implemented on the GPU")
    lib = load_library("gpu")
    d = _as_device(x, torch.float32)
    if d.ndim != 1:
        raise ValueError("x must be one-dimensional")
    if distance is not None and distance < 1:
        raise ValueError("`distance` must be greater or equal to 1")
    if wlen is not None and prominence is not None and math.ceil(wlen) <= 1:
        raise ValueError(f"`wlen` must be larger than 1, was {math.ceil(wlen)}")
    n = int(d.shape[0])
    cap = max(n // 2, 1)
    opt = PeakOptions()
    opt.distance = 0.0 if distance is None else float(distance)
    keep_alive = []
    for name, cond in (("height", height), ("threshold", threshold),
                       ("prominence", prominence)):
        if cond is None:
            setattr(opt, f"{name}_min", float("nan"))
            setattr(opt, f"{name}_max", float("nan"))
            continue
        setattr(opt, f"use_{name}", 1)
        lo, hi, lo_a, hi_a = _borders(cond, n, d.device)
        keep_alive += [lo_a, hi_a]
        setattr(opt, f"{name}_min", lo)
        setattr(opt, f"{name}_max", hi)
        setattr(opt, f"d_{name}_min", None if lo_a is None else lo_a.data_ptr())
        setattr(opt, f"d_{name}_max", None if hi_a is None else hi_a.data_ptr())
    opt.wlen = 0.0 if wlen is None else float(wlen)
    peaks = torch.empty(cap, dtype=torch.int32, device=d.device)
    prom = lb = rb = None
    if prominence is not None:
        prom = torch.empty(cap, dtype=torch.float64, device=d.device)
        lb = torch.empty(cap, dtype=torch.int32, device=d.device)
        rb = torch.empty(cap, dtype=torch.int32, device=d.device)
    count = ct.c_size_t(0)
    from .tables import _stream_ptr
    ptr = (lambda t: None if t is None else t.data_ptr())  # noqa: E731
    with torch.cuda.device(d.device):
        check(lib.bp_find_peaks_opt_dev(d.data_ptr(), n, ct.byref(opt), peaks.data_ptr(),
                                        ptr(prom), ptr(lb), ptr(rb), cap, ct.byref(count),
                                        _stream_ptr()))
    k = count.value
    p = peaks[:k].to(torch.int64)
    props = {}
    if height is not None:
        props["peak_heights"] = d[p].to(torch.float64)
    if threshold is not None:
        # the rises of the kept peaks, exact float64 differences as SciPy's
        xp = d[p].to(torch.float64)
        props["left_thresholds"] = xp - d[p - 1].to(torch.float64)
        props["right_thresholds"] = xp - d[p + 1].to(torch.float64)
    if prominence is not None:
        props["prominences"] = prom[:k]
        props["left_bases"] = lb[:k].to(torch.int64)
        props["right_bases"] = rb[:k].to(torch.int64)
    return _out(p, x), {key: _out(v, x) for key, v in props.items()}


@dataclass
class Detections:
    """Detected events: sample indexes, beam heights, winning sources
    (None without ``beam_argmax``) and the threshold used."""

    peaks: object
    heights: object
    sources: object
    threshold: object


def detect(beam_max, beam_argmax=None, threshold=None, distance=None, **threshold_kwargs):
    """Detections of the tutorial (notebooks/3_beampower.ipynb:618-626): the
    peaks of ``beam_max`` at least ``distance`` samples apart whose height is
    strictly above ``threshold``.  Without ``threshold``, it is computed by
    ``time_dependent_threshold(beam_max, **threshold_kwargs)``."""
    lib = load_library("gpu")
    bm = _as_device(beam_max, torch.float32)
    if threshold is None:
        thr = _as_device(time_dependent_threshold(bm, **threshold_kwargs), torch.float32)
    else:
        thr = _as_device(threshold, torch.float32)
    if bm.ndim != 1 or thr.shape != bm.shape:
        raise ValueError("beam_max and threshold must be one-dimensional and of one length")
    if distance is not None and distance < 1:
        raise ValueError("`distance` must be greater or equal to 1")
    am = None if beam_argmax is None else _as_device(beam_argmax, torch.int32)
    n = int(bm.shape[0])
    cap = max(n // 2, 1)
    peaks = torch.empty(cap, dtype=torch.int32, device=bm.device)
    heights = torch.empty(cap, dtype=torch.float32, device=bm.device)
    sources = torch.empty(cap, dtype=torch.int32, device=bm.device) if am is not None else None
    count = ct.c_size_t(0)
    from .tables import _stream_ptr
    with torch.cuda.device(bm.device):
        check(lib.bp_detect_dev(bm.data_ptr(), None if am is None else am.data_ptr(),
                                thr.data_ptr(), n, 0.0 if distance is None else float(distance),
                                peaks.data_ptr(), heights.data_ptr(),
                                None if sources is None else sources.data_ptr(), cap,
                                ct.byref(count), _stream_ptr()))
    k = count.value
    return Detections(peaks=_out(peaks[:k].to(torch.int64), beam_max),
                      heights=_out(heights[:k], beam_max),
                      sources=None if sources is None else _out(sources[:k].to(torch.int64),
                                                                beam_max),
                      threshold=_out(thr, beam_max) if threshold is None else threshold)
