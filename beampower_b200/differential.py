"""Differential beamforming on the GPU (beampower/src/beamform.c:338-394).

The reference computes it on the CPU only; its GPU branch prints "not yet
implemented" (beampower/beampower.py:220-223).  Here the channel prestack and
the per-source beam at the zero lag both run on the GPU.
"""
from __future__ import annotations

import numpy as np

from .core import check, load_library


def beamform_differential(waveform_features, time_delays, weights_phases, weights_sources):
    """(n_sources,) float32 beams at the zero lag (n_samples - 1) // 2 of
    inter-station correlation features, strict rule; sources the rule
    rejects keep 0."""
    from .beampower import _is_cuda_tensor, prestack_traces
    lib = load_library("gpu")
    if _is_cuda_tensor(waveform_features) or _is_cuda_tensor(time_delays):
        import torch
        from .tables import _dev_tensor, _stream_ptr
        dev = waveform_features.device if _is_cuda_tensor(waveform_features) else \
            time_delays.device
        F = _dev_tensor(waveform_features, torch.float32, dev)
        A = _dev_tensor(weights_phases, torch.float32, dev)
        D = _dev_tensor(time_delays, torch.int32, dev)
        W = _dev_tensor(weights_sources, torch.float32, dev)
        S, C, T = map(int, F.shape)
        N, _, P = map(int, D.shape)
        rows = torch.empty((S * P, max(T, 1)), dtype=torch.float32, device=dev)
        check(lib.bp_prestack_dev(F.data_ptr(), A.data_ptr(), T, S, C, P, 0, 0, max(T, 1),
                                  rows.data_ptr(), None, _stream_ptr()))
        beam = torch.zeros(N, dtype=torch.float32, device=dev)
        check(lib.bp_beamform_differential_dev(rows.data_ptr(), T, 0, max(T, 1), D.data_ptr(),
                                               W.data_ptr(), N, S, P, beam.data_ptr(),
                                               _stream_ptr()))
        return beam
    U = prestack_traces(waveform_features, weights_phases)
    D = np.ascontiguousarray(time_delays, dtype=np.int32)
    W = np.ascontiguousarray(weights_sources, dtype=np.float32)
    S, T, P = U.shape
    N = D.shape[0]
    beam = np.zeros(N, dtype=np.float32)
    fn = lib.beamform_differential
    check(fn(U.ctypes.data_as(fn.argtypes[0]), D.ctypes.data_as(fn.argtypes[1]),
             W.ctypes.data_as(fn.argtypes[2]), T, N, S, P, 0, beam.ctypes.data_as(fn.argtypes[8])))
    return beam
