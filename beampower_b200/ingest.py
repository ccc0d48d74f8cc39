"""Travel times in seconds to sample delays, on the GPU.

The reference tutorial reads a travel-time grid (seconds, float32, per
source, station and phase) and converts it with ``sec_to_samp``
(notebooks/3_beampower.ipynb:378-394) into the int32 ``time_delays`` that
``beamform`` takes, optionally relative to each source's earliest arrival
(:396).  ``sec_to_samp`` here gives identical integers; reading the
tutorial's HDF5 file stays with the caller.
"""
from __future__ import annotations

from .core import check, load_library

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def sec_to_samp(t, sr, epsilon=0.2, relative=False):
    """int32 sample delays of travel times ``t`` (seconds) at rate ``sr``:
    sign(t) * trunc(|t * sr| + epsilon) in float32, as the tutorial.

    relative: subtract each source's smallest delay (t shaped (N, S, P)).
    numpy in, numpy out; tensor in, tensor out."""
    from .tables import _dev_tensor, _stream_ptr
    if torch is None:
        raise RuntimeError("torch is required for sec_to_samp")
    lib = load_library("gpu")
    is_tensor = isinstance(t, torch.Tensor)
    dev = t.device if is_tensor and t.is_cuda else torch.device("cuda",
                                                                torch.cuda.current_device())
    x = _dev_tensor(t, torch.float32, dev)
    if relative and x.ndim != 3:
        raise ValueError("relative delays need travel times shaped (sources, stations, phases)")
    n_src = int(x.shape[0]) if x.ndim else 1
    per = int(x.numel() // n_src) if n_src else 0
    out = torch.empty(x.shape, dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        check(lib.bp_seconds_to_samples_dev(x.data_ptr(), n_src, per, float(sr), float(epsilon),
                                            1 if relative else 0, out.data_ptr(), _stream_ptr()))
    return out if is_tensor else out.cpu().numpy()
