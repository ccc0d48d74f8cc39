"""Batch scheduler: many detection windows in one persistent launch.

Each window has its own length and station subset and uses one of a few
resident travel-time tables.  The windows' traces are prestacked on the GPU
into per-window buffers, then one persistent kernel beamforms all of them,
popping work items (window, source tile, 4096-sample time chunk) from a
device work queue, and one kernel decodes every window's max/argmax.  The
whole step -- prestack of every window, queue reset, persistent launch,
decode -- is stream-ordered device work, so it is captured once in a CUDA
graph and replayed for every new set of window data copied into the same
input buffers.

The reference runs one ``beamform`` call per window
(beampower/beampower.py:10-227); a window's station subset is expressed there
by zeroing columns of ``weights_sources``.  Here the subset is a station mask
on a shared table, with the strict rule's delay range recomputed for it.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np

from .core import STORAGE, Record, check, load_library, trace_copies
from .tables import _dev_tensor, _stream_ptr

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


@dataclass
class Window:
    """One detection window.

    table: index into the batch's tables
    n_samples: record length
    stations: station indexes the window uses (None: all)
    out_of_bounds: 'strict' or 'flexible'
    """

    table: int
    n_samples: int
    stations: object = None
    out_of_bounds: str = "strict"


def station_mask_words(stations, n_stations):
    """Bit mask (uint32 words) of a station subset; bit s set = station used."""
    words = np.zeros((n_stations + 31) // 32, dtype=np.uint32)
    if stations is None:
        stations = range(n_stations)
    for s in stations:
        if not 0 <= int(s) < n_stations:
            raise ValueError(f"station {s} outside 0..{n_stations - 1}")
        words[int(s) >> 5] |= np.uint32(1) << np.uint32(int(s) & 31)
    return words


class WindowBatch:
    """A fixed layout of windows over resident tables.

    Parameters
    ----------
    tables: list of TravelTimeTable (same n_phases, same device)
    windows: list of Window
    weights_phases: (S, C, P) channel -> phase weights shared by the windows
    storage: 'fp16' (default), 'fp32' or 'bf16'.  FP16 storage halves the
        trace bytes and stays within 1e-3 of a float64 beam (11 significant
        bits: at most two roundings of 2^-11 per term of one sign); FP32
        gives the reference's bits; BF16 (8 significant bits) cannot promise
        1e-3 (one rounding alone is up to 2^-8 = 3.9e-3).  A table whose
        delay windows are too wide for the four 16-bit copies of every
        window in any kernel shape, while its FP32 windows fit one, makes
        the batch store FP32 (``self.storage`` says which): those traces
        take half the bytes of the 16-bit copies, run at the same speed and
        give the reference's bits.
    """

    def __init__(self, tables, windows, weights_phases, storage="fp16", stream=None):
        if torch is None:
            raise RuntimeError("torch is required for batches")
        self.lib = load_library("gpu")
        self.tables = list(tables)
        self.windows = list(windows)
        self.device = self.tables[0].device
        st = STORAGE[storage]
        if st != 0 and any(self.lib.bp_table_kernel_config(t.handle, st, 1) < 0
                           and self.lib.bp_table_kernel_config(t.handle, 0, 1) >= 0
                           for t in self.tables):
            storage, st = "fp32", 0
        self.storage = storage
        P = self.tables[0].n_phases
        self.alpha = _dev_tensor(weights_phases, torch.float32, self.device)
        S, C, _ = self.alpha.shape
        self.n_channels = C
        elem = torch.float32 if st == 0 else (torch.bfloat16 if st == 1 else torch.float16)
        self.features, self.traces, self.scales = [], [], []
        self.masks, self.beam_max, self.argmax, self.layouts = [], [], [], []
        recs = (Record * len(self.windows))()
        for i, w in enumerate(self.windows):
            tab = self.tables[w.table]
            if tab.n_stations != S or tab.n_phases != P:
                raise ValueError("window tables must match weights_phases")
            lpad, pitch = tab.layout(w.n_samples)
            rows = S * P * trace_copies(st)
            self.features.append(torch.zeros((S, C, w.n_samples), dtype=torch.float32,
                                             device=self.device))
            self.traces.append(torch.empty((rows, pitch), dtype=elem, device=self.device))
            self.scales.append(torch.ones(S, dtype=torch.float32, device=self.device))
            self.beam_max.append(torch.zeros(w.n_samples, dtype=torch.float32,
                                             device=self.device))
            self.argmax.append(torch.zeros(w.n_samples, dtype=torch.int32, device=self.device))
            self.layouts.append((lpad, pitch))
            mask = None
            if w.stations is not None:
                mask = torch.from_numpy(station_mask_words(w.stations, S).view(np.int32)).to(
                    self.device)
            self.masks.append(mask)
            r = recs[i]
            r.table = w.table
            r.out_of_bounds = 0 if w.out_of_bounds == "strict" else 1
            r.traces = self.traces[-1].data_ptr()
            r.scales = self.scales[-1].data_ptr()
            r.n_samples = w.n_samples
            r.lpad = lpad
            r.pitch = pitch
            r.t_origin = 0
            r.out0 = 0
            r.out1 = w.n_samples
            r.station_mask = mask.data_ptr() if mask is not None else None
            r.beam_max = self.beam_max[-1].data_ptr()
            r.argmax = self.argmax[-1].data_ptr()
        tabs = (ct.c_void_p * len(self.tables))(*[t.handle.value for t in self.tables])
        handle = ct.c_void_p()
        check(self.lib.bp_batch_create(tabs, len(self.tables), recs, len(self.windows), st,
                                       _stream_ptr(stream), ct.byref(handle)))
        self.handle = handle
        self._st = st
        self.graph = None

    # ------------------------------------------------------------------
    def set_features(self, i, waveform_features):
        """Copy new (S, C, T_i) features of window i into its input buffer."""
        src = waveform_features
        if isinstance(src, np.ndarray):
            src = torch.from_numpy(np.ascontiguousarray(src, dtype=np.float32))
        self.features[i].copy_(src, non_blocking=True)

    def _step(self, stream):
        sp = _stream_ptr(stream)
        S, C, P = self.alpha.shape
        for bm in self.beam_max:  # a fresh call's zeroed outputs (beampower.py:175)
            bm.zero_()
        for i, w in enumerate(self.windows):
            lpad, pitch = self.layouts[i]
            check(self.lib.bp_prestack_dev(self.features[i].data_ptr(), self.alpha.data_ptr(),
                                           w.n_samples, S, C, P, self._st, lpad, pitch,
                                           self.traces[i].data_ptr(),
                                           self.scales[i].data_ptr(), sp))
        check(self.lib.bp_batch_run(self.handle, sp))

    def run(self, stream=None):
        """Prestack every window and beamform the batch (stream-ordered)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._step(stream)
        return self.results()

    def capture(self):
        """Record one step (all prestacks + the batch launch) in a CUDA graph;
        later ``run()`` calls replay it."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._step(s)  # warm-up outside capture (attributes, lazy loading)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._step(torch.cuda.current_stream())
        self.graph = g
        return g

    def results(self):
        """[(beam_max, argmax)] CUDA tensors, one pair per window."""
        return list(zip(self.beam_max, self.argmax))

    def status(self, stream=None):
        v = ct.c_int(0)
        check(self.lib.bp_batch_status(self.handle, _stream_ptr(stream), ct.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "handle", None):
            self.graph = None
            self.lib.bp_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def terms(self):
        """Nominal beam terms of one step: sum of N x T x S_window x P."""
        total = 0
        for w in self.windows:
            tab = self.tables[w.table]
            n_sta = tab.n_stations if w.stations is None else len(list(w.stations))
            total += tab.n_sources * w.n_samples * n_sta * tab.n_phases
        return total
