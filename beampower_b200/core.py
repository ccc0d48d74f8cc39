"""ctypes loader of the sm_100a library, mirroring beampower/core.py.

The reference keeps a per-device table of shared objects and their argtypes
(beampower/core.py:9-89) and a loader that loads each one once and caches it
(core.py:92-169).  This module does the same for the single GPU library this
package ships, ``lib/libbeampower_b200.so``.  The ``"gpu"`` entry binds the
reference GPU symbols with the reference argtypes (core.py:65-87) plus the
device-pointer entry points of include/beampower_b200.h.

There is no ``"cpu"`` entry: this package is the GPU path.  The product path
never falls back to a CPU implementation; if the library is missing,
``load_library("gpu")`` raises like the reference does (core.py:156-163).
"""
from __future__ import annotations

import ctypes as ct
import os

DIRPATH_LIBRARIES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

_f32p = ct.POINTER(ct.c_float)
_i32p = ct.POINTER(ct.c_int)
_vp = ct.c_void_p
_sz = ct.c_size_t
_int = ct.c_int


class TableInfo(ct.Structure):
    """Mirror of ``bp_table_info`` (include/beampower_b200.h)."""

    _fields_ = [
        ("n_sources", ct.c_int64),
        ("n_stations", ct.c_int64),
        ("n_phases", ct.c_int64),
        ("tile_sources", ct.c_int32),
        ("n_tiles", ct.c_int32),
        ("min_delay", ct.c_int32),
        ("max_delay", ct.c_int32),
        ("max_spread", ct.c_int32),
        ("max_active", ct.c_int32),
        ("any_nonfinite", ct.c_int32),
        ("uses_window_kernel", ct.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Record(ct.Structure):
    """Mirror of ``bp_record`` (include/beampower_b200.h)."""

    _fields_ = [
        ("table", ct.c_int32),
        ("out_of_bounds", ct.c_int32),
        ("traces", ct.c_void_p),
        ("scales", ct.c_void_p),
        ("n_samples", ct.c_size_t),
        ("lpad", ct.c_size_t),
        ("pitch", ct.c_size_t),
        ("t_origin", ct.c_int64),
        ("out0", ct.c_size_t),
        ("out1", ct.c_size_t),
        ("station_mask", ct.c_void_p),
        ("beam_max", ct.c_void_p),
        ("argmax", ct.c_void_p),
    ]


class PeakOptions(ct.Structure):
    """bp_peak_options (include/beampower_b200.h)."""

    _fields_ = [
        ("distance", ct.c_double),
        ("use_height", ct.c_int32),
        ("height_min", ct.c_double),
        ("height_max", ct.c_double),
        ("d_height_min", ct.c_void_p),
        ("d_height_max", ct.c_void_p),
        ("use_threshold", ct.c_int32),
        ("threshold_min", ct.c_double),
        ("threshold_max", ct.c_double),
        ("d_threshold_min", ct.c_void_p),
        ("d_threshold_max", ct.c_void_p),
        ("use_prominence", ct.c_int32),
        ("prominence_min", ct.c_double),
        ("prominence_max", ct.c_double),
        ("d_prominence_min", ct.c_void_p),
        ("d_prominence_max", ct.c_void_p),
        ("wlen", ct.c_double),
    ]


# symbol -> (argtypes, restype)
SIGNATURES = {
    # drop-ins, argtypes of beampower/core.py:65-87 (restype added: int status)
    "beamform": ([_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, _int, _f32p], _int),
    "beamform_max": ([_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, _int, _f32p, _i32p], _int),
    # CPU-library prototype of the prestack (core.py:50-59), run on the GPU
    "prestack_waveform_features": ([_f32p, _f32p, _sz, _sz, _sz, _sz, _int, _f32p], _int),
    "bp_beamform_host": ([_vp, _vp, _vp, _vp, _sz, _sz, _sz, _sz, _sz, _int, _int, _int,
                          _vp, _vp, _vp], _int),
    "bp_table_create": ([_vp, _vp, _sz, _sz, _sz, _vp, ct.POINTER(_vp)], _int),
    "bp_table_destroy": ([_vp], _int),
    "bp_table_get_info": ([_vp, ct.POINTER(TableInfo)], _int),
    "bp_trace_layout": ([_vp, _sz, ct.POINTER(_sz), ct.POINTER(_sz)], _int),
    "bp_prestack_dev": ([_vp, _vp, _sz, _sz, _sz, _sz, _int, _sz, _sz, _vp, _vp, _vp], _int),
    "bp_traces_from_prestacked_dev": ([_vp, _sz, _sz, _sz, _sz, _sz, _vp, _vp], _int),
    "bp_beamform_max_dev": ([_vp, _vp, _int, _vp, _sz, _sz, _sz, _int, _vp, _vp, _vp, _vp],
                            _int),
    "bp_beamform_dev": ([_vp, _vp, _int, _vp, _sz, _sz, _sz, _int, _vp, _sz, _vp], _int),
    "bp_minmax_dev": ([_vp, _vp, _sz, _sz, _sz, _vp, _vp], _int),
    "bp_beamform_max_direct_dev": ([_vp, _int, _vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, _sz,
                                    _int, _vp, _vp, _vp, _vp], _int),
    "beamform_differential": ([_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, _int, _f32p], _int),
    "bp_beamform_differential_dev": ([_vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, _sz, _vp, _vp],
                                     _int),
    "bp_threshold_dev": ([_vp, _sz, _sz, ct.c_double, _int, ct.c_float, _vp, _sz,
                          ct.c_ulonglong, _vp, _vp], _int),
    "bp_find_peaks_dev": ([_vp, _sz, ct.c_double, _vp, _sz, ct.POINTER(_sz), _vp], _int),
    "bp_find_peaks_opt_dev": ([_vp, _sz, ct.POINTER(PeakOptions), _vp, _vp, _vp, _vp, _sz,
                               ct.POINTER(_sz), _vp], _int),
    "bp_detect_dev": ([_vp, _vp, _vp, _sz, ct.c_double, _vp, _vp, _vp, _sz, ct.POINTER(_sz),
                       _vp], _int),
    "bp_pairwise_sum_f32": ([_vp, _sz], ct.c_float),
    "bp_trace_copies": ([_int], _int),
    "bp_keys_to_shared_dev": ([_vp, _sz, _sz, _vp], _int),
    "bp_keys_from_shared_dev": ([_vp, _sz, _vp, _vp, _vp], _int),
    "bp_envelope_dev": ([_vp, _sz, _sz, ct.c_float, _vp, _vp], _int),
    "bp_seconds_to_samples_dev": ([_vp, _sz, _sz, ct.c_double, ct.c_double, _int, _vp, _vp],
                                  _int),
    "bp_prestack_envelope_dev": ([_vp, _vp, _sz, _sz, _sz, _sz, ct.c_float, _int, _sz, _sz, _vp,
                                  _vp, _vp], _int),
    "bp_measure_peaks": ([_vp, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], _int),
    "bp_beamform_max_noalloc": ([_vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, _sz, _int, _vp, _vp,
                                 _vp], _int),
    "bp_batch_create": ([ct.POINTER(_vp), _int, ct.POINTER(Record), _int, _int, _vp,
                         ct.POINTER(_vp)], _int),
    "bp_batch_run": ([_vp, _vp], _int),
    "bp_record_beamform_max_dev": ([_vp, ct.POINTER(Record), _int, _vp, _vp], _int),
    "bp_batch_status": ([_vp, _vp, ct.POINTER(_int)], _int),
    "bp_batch_destroy": ([_vp], _int),
    "bp_kernel_config_count": ([], _int),
    "bp_kernel_config_describe": ([_int, ct.POINTER(_int), ct.POINTER(_int), ct.POINTER(_int),
                                   ct.POINTER(_int)], _int),
    "bp_kernel_config_shape": ([_int, ct.POINTER(_int), ct.POINTER(_int), ct.POINTER(_int)],
                               _int),
    "bp_set_kernel_config": ([_int, _int, _int], _int),
    "bp_get_kernel_config": ([_int, _int], _int),
    "bp_table_kernel_config": ([_vp, _int, _int], _int),
    "bp_debug_wait_timeout": ([ct.c_ulonglong, _vp, ct.POINTER(_int)], _int),
    "bp_last_error": ([], ct.c_char_p),
    "bp_version": ([], ct.c_char_p),
    "bp_launch_count": ([], ct.c_uint64),
}

LIBRARIES = {
    "gpu": {
        "filepath_library": os.path.join(DIRPATH_LIBRARIES, "libbeampower_b200.so"),
        "is_loaded": False,
        "lib": None,
        "beamform_argtypes": SIGNATURES["beamform"][0],
        "beamform_max_argtypes": SIGNATURES["beamform_max"][0],
    },
}

# Status codes of include/beampower_b200.h
BP_OK = 0
STATUS_NAMES = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
                4: "unsupported shape", 5: "kernel failure",
                6: "beyond the fixed scratch limit of the allocation-free entry point "
                   "(524288 samples, 524288 sources)"}
STORAGE = {"fp32": 0, "f32": 0, "float32": 0, "bf16": 1, "bfloat16": 1, "fp16": 2,
           "f16": 2, "float16": 2}
REDUCE_NONE, REDUCE_MAX = 0, 1


class BeampowerError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"beampower_b200: {STATUS_NAMES.get(status, status)}: {message}")


def load_library(device: str = "gpu"):
    """Load the library for ``device`` once and cache it (beampower/core.py:92-169).

    Raises
    ------
    NameError
        ``device`` is not ``"gpu"`` (this package has no CPU library).
    RuntimeError
        The GPU shared object has not been built.
    """
    device_name = device.lower()
    if device_name not in LIBRARIES:
        raise NameError(
            f"Device should be gpu, not {device_name} (beampower_b200 implements the GPU "
            "path only; the CPU path is the reference package's)")
    info = LIBRARIES[device_name]
    if info["is_loaded"]:
        return info["lib"]
    # BEAMPOWER_B200_LIBRARY selects another build of the library, e.g. the
    # index-checked one (lib/libbeampower_b200_checked.so)
    path = os.environ.get("BEAMPOWER_B200_LIBRARY") or info["filepath_library"]
    if not os.path.exists(path):
        raise RuntimeError(
            f"GPU library not available. The shared object {path} does not exist.\n"
            "Build it with `python -m beampower_b200.build` (nvcc, sm_100a).")
    lib = ct.CDLL(path)
    for name, (argtypes, restype) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    info["is_loaded"] = True
    info["lib"] = lib
    return lib


def check(status: int) -> None:
    """Raise BeampowerError for a non-zero status, with the library's message."""
    if status != BP_OK:
        lib = load_library("gpu")
        msg = lib.bp_last_error()
        raise BeampowerError(status, msg.decode() if msg else "")


def launch_count() -> int:
    """Kernel launches issued by the library in this process."""
    return int(load_library("gpu").bp_launch_count())


def trace_copies(storage: int) -> int:
    """Rows per (station, phase) of trace storage (1 FP32, 4 for 16-bit)."""
    n = load_library("gpu").bp_trace_copies(int(storage))
    if n < 1:
        raise ValueError(f"unknown storage {storage}")
    return n
