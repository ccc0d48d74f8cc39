"""Waveform features on the GPU: the tutorial's envelope transform.

notebooks/3_beampower.ipynb:74-103 defines ``envelope(x)``: the modulus of
the analytic signal (scipy.signal.hilbert), minus its median, divided by its
median absolute deviation (1 when that is 0), clipped above at 1e5; the
tutorial applies it to every (station, channel) trace (:145-147) to make the
``waveform_features`` that ``beamform`` takes.  Here every row goes through
cuFFT and the library's own kernels in one device call; results match the
tutorial to float32 FFT rounding.

``TravelTimeTable.traces_from_waveforms`` goes one step further: raw
waveforms straight to the beamformer's trace rows.

Inputs are converted to float32 first.  The tutorial's traces may be
float64 (as ObsPy reads them), in which case SciPy computes their envelope in
float64 before the float32 feature array stores it; the float32 FFTs here
then differ from it by float32 rounding, within the same bound as from the
float32 tutorial path.
"""
from __future__ import annotations

from .core import check, load_library

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def envelope(x, clip_max=1e5):
    """Envelope feature of every row of x (..., T): same shape, float32.

    numpy in, numpy out; tensor in, tensor out (CUDA tensors stay on their
    device)."""
    from .tables import _dev_tensor, _stream_ptr
    if torch is None:
        raise RuntimeError("torch is required for the feature functions")
    lib = load_library("gpu")
    is_tensor = isinstance(x, torch.Tensor)
    dev = x.device if is_tensor and x.is_cuda else torch.device("cuda",
                                                                torch.cuda.current_device())
    d = _dev_tensor(x, torch.float32, dev)
    if d.ndim == 0:
        raise ValueError("x must have at least one dimension")
    T = int(d.shape[-1])
    rows = int(d.numel() // T) if T else 0
    out = torch.empty_like(d)
    with torch.cuda.device(dev):
        check(lib.bp_envelope_dev(d.data_ptr(), rows, T, float(clip_max), out.data_ptr(),
                                  _stream_ptr()))
    return out if is_tensor else out.cpu().numpy()


def waveform_features(waveforms, clip_max=1e5):
    """(S, C, T) waveforms -> (S, C, T) envelope features (the tutorial's
    feature loop, notebooks/3_beampower.ipynb:145-147)."""
    return envelope(waveforms, clip_max)
