"""Resident travel-time tables and device-side calls on torch tensors.

A ``TravelTimeTable`` uploads (or adopts) ``time_delays`` and
``weights_sources`` once and keeps the library's tiled table in HBM, so that
every later call on new waveform data only moves the traces.  This is the
object the batch and stream schedulers hold per network.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from .core import STORAGE, TableInfo, check, load_library, trace_copies

try:  # torch is plumbing (device memory, streams), imported lazily where needed
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _require_torch():
    if torch is None:
        raise RuntimeError("torch is required for device-resident tables")


def _stream_ptr(stream=None) -> int:
    _require_torch()
    s = torch.cuda.current_stream() if stream is None else stream
    return int(s.cuda_stream)


def _dev_tensor(x, dtype, device):
    """Contiguous CUDA tensor of ``dtype`` (copying host data if needed)."""
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x))
    if not isinstance(x, torch.Tensor):
        x = torch.as_tensor(x)
    return x.to(device=device, dtype=dtype).contiguous()


class TravelTimeTable:
    """Device-resident (time_delays, weights_sources) pair.

    Parameters
    ----------
    time_delays: (n_sources, n_stations, n_phases) int array or tensor
    weights_sources: (n_sources, n_stations) float array or tensor
    device: torch device (default: current CUDA device)
    """

    def __init__(self, time_delays, weights_sources, device=None, stream=None):
        _require_torch()
        self.lib = load_library("gpu")
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else \
            torch.device(device)
        self.device = dev
        with torch.cuda.device(dev):
            self.delays = _dev_tensor(time_delays, torch.int32, dev)
            self.weights = _dev_tensor(weights_sources, torch.float32, dev)
            if self.delays.dim() != 3 or self.weights.dim() != 2 or \
                    self.weights.shape != self.delays.shape[:2]:
                raise ValueError("time_delays must be (N, S, P) and weights_sources (N, S)")
            self.n_sources, self.n_stations, self.n_phases = map(int, self.delays.shape)
            handle = ct.c_void_p()
            check(self.lib.bp_table_create(self.delays.data_ptr(), self.weights.data_ptr(),
                                           self.n_sources, self.n_stations, self.n_phases,
                                           _stream_ptr(stream), ct.byref(handle)))
            self.handle = handle
        info = TableInfo()
        check(self.lib.bp_table_get_info(self.handle, ct.byref(info)))
        self.info = info.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            self.lib.bp_table_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self, n_samples: int):
        """(lpad, pitch) of trace storage for a record of ``n_samples``."""
        lpad, pitch = ct.c_size_t(), ct.c_size_t()
        check(self.lib.bp_trace_layout(self.handle, int(n_samples), ct.byref(lpad),
                                       ct.byref(pitch)))
        return int(lpad.value), int(pitch.value)

    # ------------------------------------------------------------------
    def traces_from_features(self, waveform_features, weights_phases, storage="fp32",
                             stream=None):
        """GPU prestack of (S, C, T) features into this table's trace layout.

        Returns a ``Traces`` record (device buffer + layout)."""
        F = _dev_tensor(waveform_features, torch.float32, self.device)
        A = _dev_tensor(weights_phases, torch.float32, self.device)
        S, C, T = map(int, F.shape)
        if S != self.n_stations or A.shape != (S, C, self.n_phases):
            raise ValueError("waveform_features / weights_phases do not match the table")
        st = STORAGE[storage]
        lpad, pitch = self.layout(T)
        elem = torch.float32 if st == 0 else (torch.bfloat16 if st == 1 else torch.float16)
        # 16-bit storage keeps shifted copies of every row so that any run of
        # 4 samples is one aligned 64-bit word pair (trace_copies rows per row)
        rows = S * self.n_phases * trace_copies(st)
        buf = torch.empty((rows, pitch), dtype=elem, device=self.device)
        scales = torch.ones(S, dtype=torch.float32, device=self.device)
        check(self.lib.bp_prestack_dev(F.data_ptr(), A.data_ptr(), T, S, C, self.n_phases, st,
                                       lpad, pitch, buf.data_ptr(), scales.data_ptr(),
                                       _stream_ptr(stream)))
        return Traces(buf, scales, st, T, lpad, pitch)

    @classmethod
    def from_travel_times(cls, travel_times, sampling_rate, weights_sources, epsilon=0.2,
                          relative=False, device=None):
        """Table from travel times in seconds (N, S, P): the tutorial's
        sec_to_samp conversion (notebooks/3_beampower.ipynb:378-396) on the
        device, then the table build."""
        from .ingest import sec_to_samp
        _require_torch()
        dev = device if device is not None else torch.device("cuda",
                                                             torch.cuda.current_device())
        tt = _dev_tensor(travel_times, torch.float32, dev)
        return cls(sec_to_samp(tt, sampling_rate, epsilon, relative), weights_sources,
                   device=dev)

    def traces_from_waveforms(self, waveforms, weights_phases, storage="fp32", clip_max=1e5,
                              stream=None):
        """Raw (S, C, T) waveforms to this table's trace layout in one device
        call: the tutorial's envelope feature of every (station, channel)
        (notebooks/3_beampower.ipynb:74-103) and then the prestack."""
        X = _dev_tensor(waveforms, torch.float32, self.device)
        A = _dev_tensor(weights_phases, torch.float32, self.device)
        S, C, T = map(int, X.shape)
        if S != self.n_stations or A.shape != (S, C, self.n_phases):
            raise ValueError("waveforms / weights_phases do not match the table")
        st = STORAGE[storage]
        lpad, pitch = self.layout(T)
        elem = torch.float32 if st == 0 else (torch.bfloat16 if st == 1 else torch.float16)
        rows = S * self.n_phases * trace_copies(st)
        buf = torch.empty((rows, pitch), dtype=elem, device=self.device)
        scales = torch.ones(S, dtype=torch.float32, device=self.device)
        check(self.lib.bp_prestack_envelope_dev(X.data_ptr(), A.data_ptr(), T, S, C,
                                                self.n_phases, float(clip_max), st, lpad, pitch,
                                                buf.data_ptr(), scales.data_ptr(),
                                                _stream_ptr(stream)))
        return Traces(buf, scales, st, T, lpad, pitch)

    def traces_from_prestacked(self, prestacked, stream=None):
        """(S, T, P) prestacked float32 traces -> this table's layout."""
        U = _dev_tensor(prestacked, torch.float32, self.device)
        S, T, P = map(int, U.shape)
        if S != self.n_stations or P != self.n_phases:
            raise ValueError("prestacked traces do not match the table")
        lpad, pitch = self.layout(T)
        buf = torch.empty((S * P, pitch), dtype=torch.float32, device=self.device)
        check(self.lib.bp_traces_from_prestacked_dev(U.data_ptr(), T, S, P, lpad, pitch,
                                                     buf.data_ptr(), _stream_ptr(stream)))
        return Traces(buf, None, 0, T, lpad, pitch)

    # ------------------------------------------------------------------
    def beamform_max(self, traces, out_of_bounds=0, stream=None, out=None):
        """Max / argmax over sources; returns (beam_max, argmax) CUDA tensors."""
        T = traces.n_samples
        if out is None:
            beam_max = torch.zeros(T, dtype=torch.float32, device=self.device)
            argmax = torch.zeros(T, dtype=torch.int32, device=self.device)
            keys = torch.empty(max(T, 1), dtype=torch.int64, device=self.device)
        else:
            beam_max, argmax, keys = out
        scales = traces.scales.data_ptr() if traces.scales is not None else None
        check(self.lib.bp_beamform_max_dev(self.handle, traces.buf.data_ptr(), traces.storage,
                                           scales, T, traces.lpad, traces.pitch,
                                           int(out_of_bounds), keys.data_ptr(),
                                           beam_max.data_ptr(), argmax.data_ptr(),
                                           _stream_ptr(stream)))
        return beam_max, argmax

    def beamform(self, traces, out_of_bounds=0, stream=None, out=None):
        """Full (n_sources, n_samples) response as a CUDA tensor."""
        T = traces.n_samples
        beam = torch.zeros((self.n_sources, T), dtype=torch.float32, device=self.device) \
            if out is None else out
        scales = traces.scales.data_ptr() if traces.scales is not None else None
        check(self.lib.bp_beamform_dev(self.handle, traces.buf.data_ptr(), traces.storage,
                                       scales, T, traces.lpad, traces.pitch,
                                       int(out_of_bounds), beam.data_ptr(), beam.stride(0),
                                       _stream_ptr(stream)))
        return beam


class Traces:
    """Prestacked traces in a table's device layout."""

    def __init__(self, buf, scales, storage, n_samples, lpad, pitch):
        self.buf = buf
        self.scales = scales
        self.storage = storage
        self.n_samples = n_samples
        self.lpad = lpad
        self.pitch = pitch

    def to_prestacked(self, n_phases):
        """Back to the reference's (S, T, P) float32 layout (for checks)."""
        buf = self.buf[0::trace_copies(self.storage)]
        rows = buf[:, self.lpad:self.lpad + self.n_samples].float()
        if self.scales is not None and self.storage != 0:
            rows = rows * self.scales.repeat_interleave(n_phases)[:, None]
        S = rows.shape[0] // n_phases
        return rows.reshape(S, n_phases, self.n_samples).permute(0, 2, 1).contiguous()
