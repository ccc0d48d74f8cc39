"""CPU restatement of the tutorial's travel-time conversion.

Test infrastructure: only the tests use this module, as the checker of the
GPU conversion.  Restates ``sec_to_samp`` of notebooks/3_beampower.ipynb:
378-394 (float32 arithmetic: the seconds are float32 and the sampling rate a
Python float) and the optional relative delays of :396.
"""
from __future__ import annotations

import numpy as np


def sec_to_samp(t, sr, epsilon=0.2, relative=False):
    t = np.asarray(t, dtype=np.float32)
    with np.errstate(invalid="ignore"):
        a = np.abs(t * np.float32(sr)) + np.float32(epsilon)
        k = a.astype(np.int32)  # x86: NaN, inf and out-of-range give INT_MIN
        out = (np.sign(t) * k).astype(np.int32)
    if relative:
        out -= np.min(out, axis=(1, 2), keepdims=True)
    return out
