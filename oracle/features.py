"""CPU restatement of the tutorial's envelope features.

Test infrastructure: only the tests and the benchmark's CPU legs use this
module, as the checker of the GPU feature path.

Restates ``envelope`` of notebooks/3_beampower.ipynb:74-103 (applied to each
trace at :145-147): the modulus of the analytic signal from
scipy.signal.hilbert, minus its median, divided by its median absolute
deviation (scipy.stats.median_abs_deviation with scale 1; 1 when it is 0),
clipped above at 1e5.  SciPy (1.18.1 in this image) is the tutorial's
dependency for the Hilbert transform and the deviation; they are called
here as the tutorial calls them, in the tutorial's float32.
"""
from __future__ import annotations

import numpy as np
from scipy import signal


def envelope(x, clip_max=1e5):
    """Envelope feature of one trace (float32, same length)."""
    x = np.abs(signal.hilbert(np.asarray(x, dtype=np.float32)))
    med = np.median(x)
    mad = np.median(np.abs(x - med))
    mad = 1.0 if mad == 0.0 else mad
    x = (x - med) / mad
    return np.minimum(x, np.float32(clip_max)).astype(np.float32)


def waveform_features(waveforms, clip_max=1e5):
    """Envelope features of (..., T) waveforms, row by row."""
    w = np.asarray(waveforms, dtype=np.float32)
    flat = w.reshape(-1, w.shape[-1])
    out = np.stack([envelope(r, clip_max) for r in flat]) if flat.shape[0] else flat.copy()
    return out.reshape(w.shape)
