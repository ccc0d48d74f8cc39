"""``beamform`` front-end, a drop-in for beampower.beamform on the GPU.

Same signature, argument meaning, shapes, dtypes and error behaviour as
beampower/beampower.py:10-227, with the GPU as the only device:

* numpy inputs: one call into the C-ABI (``bp_beamform_host``) that uploads
  the arrays, prestacks on the GPU, builds the table, beamforms and returns
  numpy outputs (``beam_max`` float32 and ``beam_argmax`` int32 of shape
  (n_samples,), or ``beam`` float32 of shape (n_sources, n_samples));
* torch CUDA tensors: the device entry points on the current stream, outputs
  are CUDA tensors of the same shapes.

Error behaviour mirrors the reference: an invalid ``out_of_bounds`` prints a
message and returns None (beampower.py:81-84); an unknown device raises
NameError and a missing library RuntimeError (core.py:122-123, 157-163); an
unknown ``mode`` -- or, as in the reference, an unknown ``reduce`` in direct
mode -- prints a message and returns 1 (beampower.py:192, 225-227).  Failures
inside the library raise ``BeampowerError`` where the reference's GPU library
called exit().
"""
from __future__ import annotations

import numpy as np

from .core import REDUCE_MAX, REDUCE_NONE, STORAGE, check, load_library

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _is_cuda_tensor(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def beamform(
    waveform_features,
    time_delays,
    weights_phases,
    weights_sources,
    device="gpu",
    reduce="max",
    mode="direct",
    out_of_bounds="strict",
    num_threads=None,
    storage="fp32",
):
    """Compute the beamformed network response on the GPU.

    Parameters follow beampower.beamform (beampower/beampower.py:10-80):

    waveform_features: (n_stations, n_channels, n_samples) float array
    time_delays: (n_sources, n_stations, n_phases) int array, in samples
    weights_phases: (n_stations, n_channels, n_phases) float array
    weights_sources: (n_sources, n_stations) float array
    device: 'gpu' (the only device of this package)
    reduce: 'max' -> (beam_max, beam_argmax); 'none' / 'None' / None -> beam
    mode: 'direct' ('normal') or 'differential'
    out_of_bounds: 'strict' or 'flexible'
    num_threads: accepted for compatibility, unused
    storage: 'fp32' (default, reference-exact), 'bf16' or 'fp16' trace storage
        with a per-station scale and FP32 accumulation.
    """
    if out_of_bounds not in ["strict", "flexible"]:
        print("out_of_bounds should be either of 'strict' or 'flexible',"
              f" not {out_of_bounds}")
        return
    oob = 0 if out_of_bounds == "strict" else 1

    lib = load_library(device)
    if storage not in STORAGE:
        raise ValueError(f"storage should be one of {sorted(set(STORAGE))}, not {storage!r}")
    st = STORAGE[storage]

    # The reference draws once from NumPy's global generator on every call
    # that gets this far, whatever the mode (beampower.py:113-114); drawing
    # here too leaves a seeded caller's later draws as they were.
    if np.random.random() < 1.0e-6:
        print("beampower to the people!")

    if mode in ["normal", "direct"]:
        if reduce in ["none", "None", None]:
            red = REDUCE_NONE
        elif reduce == "max":
            red = REDUCE_MAX
        else:
            red = None
        if red is not None:
            if _is_cuda_tensor(waveform_features) or _is_cuda_tensor(time_delays):
                return _beamform_torch(waveform_features, time_delays, weights_phases,
                                       weights_sources, red, oob, storage)
            return _beamform_numpy(lib, waveform_features, time_delays, weights_phases,
                                   weights_sources, red, oob, st)

    if mode == "differential":
        from .differential import beamform_differential
        beam = beamform_differential(waveform_features, time_delays, weights_phases,
                                     weights_sources)
        if reduce in ["none", "None", None]:
            return beam
        elif reduce == "max":
            if _is_cuda_tensor(beam):
                return beam.max(dim=0).values, beam.argmax(dim=0)
            return np.max(beam, axis=0), np.argmax(beam, axis=0)
        return None

    print(f"Mode should either be 'direct' or 'differential', not {mode}.")
    return 1


def _beamform_numpy(lib, waveform_features, time_delays, weights_phases, weights_sources,
                    red, oob, storage):
    waveform_features = np.asarray(waveform_features)
    time_delays = np.asarray(time_delays)
    n_stations, n_channels, n_samples = waveform_features.shape
    n_sources, _, n_phases = time_delays.shape
    F = np.ascontiguousarray(waveform_features, dtype=np.float32)
    A = np.ascontiguousarray(weights_phases, dtype=np.float32)
    D = np.ascontiguousarray(time_delays, dtype=np.int32)
    W = np.ascontiguousarray(weights_sources, dtype=np.float32)
    if A.shape != (n_stations, n_channels, n_phases) or W.shape != (n_sources, n_stations) \
            or D.shape[1] != n_stations:
        raise ValueError("inconsistent input shapes")
    if red == REDUCE_MAX:
        beam_max = np.zeros(n_samples, dtype=np.float32)
        beam_argmax = np.zeros(n_samples, dtype=np.int32)
        check(lib.bp_beamform_host(_ptr(F), _ptr(A), _ptr(D), _ptr(W), n_samples, n_sources,
                                   n_stations, n_channels, n_phases, oob, REDUCE_MAX, storage,
                                   _ptr(beam_max), _ptr(beam_argmax), None))
        return beam_max, beam_argmax
    beam = np.zeros((n_sources, n_samples), dtype=np.float32)
    check(lib.bp_beamform_host(_ptr(F), _ptr(A), _ptr(D), _ptr(W), n_samples, n_sources,
                               n_stations, n_channels, n_phases, oob, REDUCE_NONE, storage,
                               None, None, _ptr(beam)))
    return beam


def _beamform_torch(waveform_features, time_delays, weights_phases, weights_sources, red, oob,
                    storage):
    from .tables import TravelTimeTable
    dev = waveform_features.device if _is_cuda_tensor(waveform_features) else time_delays.device
    with torch.cuda.device(dev):
        table = TravelTimeTable(time_delays, weights_sources, device=dev)
        try:
            traces = table.traces_from_features(waveform_features, weights_phases,
                                                storage=storage)
            if red == REDUCE_MAX:
                return table.beamform_max(traces, oob)
            return table.beamform(traces, oob)
        finally:
            torch.cuda.current_stream().synchronize()
            table.close()


def prestack_traces(waveform_features, weights_phases, num_threads=None, device="gpu"):
    """Channel-wise prestack on the GPU (beampower/beampower.py:230-287).

    Returns (n_stations, n_samples, n_phases) float32, phase fastest."""
    lib = load_library(device)
    F = np.ascontiguousarray(waveform_features, dtype=np.float32)
    A = np.ascontiguousarray(weights_phases, dtype=np.float32)
    n_stations, n_channels, n_samples = F.shape
    n_phases = A.shape[2]
    out = np.zeros((n_stations, n_samples, n_phases), dtype=np.float32)
    check(lib.prestack_waveform_features(
        F.ctypes.data_as(lib.prestack_waveform_features.argtypes[0]),
        A.ctypes.data_as(lib.prestack_waveform_features.argtypes[1]),
        n_samples, n_stations, n_channels, n_phases, 0,
        out.ctypes.data_as(lib.prestack_waveform_features.argtypes[7])))
    return out
