"""beampower_b200: the beamforming hot path of beampower, rebuilt for B200.

``beamform`` keeps the signature of beampower.beamform; the work runs in
hand-written sm_100a CUDA kernels (``lib/libbeampower_b200.so``) reached
through ctypes.  See ``include/beampower_b200.h`` for the C-ABI.
"""

__all__ = ["load_library", "beamform", "prestack_traces", "TravelTimeTable"]

from .core import load_library  # noqa: E402
from .beampower import beamform, prestack_traces  # noqa: E402


def __getattr__(name):
    if name == "TravelTimeTable":
        from .tables import TravelTimeTable
        return TravelTimeTable
    raise AttributeError(name)


__version__ = "0.1.0"
