"""Stream scheduler: waveform chunks from several networks, beamformed as they
arrive, with results identical to one offline call on the whole record.

Per network (``NetworkStream``) the travel-time table and weights stay
resident in HBM and the last samples of raw features are carried from chunk
to chunk.  Output sample g needs trace samples up to g + max_delay, so after
a chunk has brought the record to t_end samples the stream emits the samples
g < t_end - max_delay: for those every (source, station, phase) term the
offline call would use is available, so the emitted beams are the offline
beams, bit for bit with FP32 storage (strict and flexible rules alike).  The
carried part is the features from (next g to emit) + min(0, min_delay) on.
``flush()`` ends the record and emits the rest with the record's true length.
``state()`` / ``restore()`` (and ``save`` / ``load`` to a file) checkpoint that
carried halo and the stream position, so a stream can resume in another
process and still give the offline results.

``StreamScheduler`` is the request loop over many networks (continuous
batching): chunks are queued on arrival and admitted, earliest deadline first
(arrival + the latency budget), while fewer than ``max_inflight`` chunks are
on the GPU and their memory fits the budget.  Chunks of different networks
overlap on the device; a network's chunks run in order (each waits for the
previous one's completion event).  With ``priorities`` the admitted chunks
run on CUDA streams of graded priority: a chunk admitted while k older chunks
are in flight gets the k-th highest priority, so the SMs serve the oldest
deadline first instead of sharing them evenly among all chunks in flight.
Latency is arrival (host clock) to the completion event of the chunk's last
kernel (device clock, mapped to the host clock once).
"""
from __future__ import annotations

import ctypes as ct
import heapq
import itertools
import time

import numpy as np

from .core import STORAGE, Record, check, load_library, trace_copies
from .tables import TravelTimeTable, _dev_tensor, _stream_ptr

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


class NetworkStream:
    """Streaming state of one network.

    Parameters
    ----------
    table: TravelTimeTable of the network (resident delays and weights)
    weights_phases: (S, C, P) channel -> phase weights
    out_of_bounds: 'strict' or 'flexible'
    storage: 'fp16' (default: within 1e-3 of a float64 beam), 'fp32' (the
        reference's bits; streamed output equals the offline call bit for
        bit) or 'bf16' (within 4e-3).  A table whose delay windows are too
        wide for the four 16-bit copies of every window in any kernel shape,
        while its FP32 windows fit one, makes the stream store FP32
        (``self.storage`` says which): half the bytes, the same speed, the
        reference's bits.
    """

    def __init__(self, table: TravelTimeTable, weights_phases, out_of_bounds="strict",
                 storage="fp16", name=None):
        if torch is None:
            raise RuntimeError("torch is required for streaming")
        self.lib = load_library("gpu")
        self.table = table
        self.name = name
        self.device = table.device
        self.alpha = _dev_tensor(weights_phases, torch.float32, self.device)
        self.S, self.C, self.P = map(int, self.alpha.shape)
        self.oob = 0 if out_of_bounds == "strict" else 1
        if (STORAGE[storage] != 0
                and self.lib.bp_table_kernel_config(table.handle, STORAGE[storage], 1) < 0
                and self.lib.bp_table_kernel_config(table.handle, 0, 1) >= 0):
            storage = "fp32"
        self.storage = storage
        self._st = STORAGE[storage]
        info = table.info
        weighted = info["min_delay"] <= info["max_delay"]
        self.lead = min(0, info["min_delay"]) if weighted else 0   # <= 0
        self.lag = max(0, info["max_delay"]) if weighted else 0    # >= 0
        self.t_end = 0     # samples received
        self.t_emit = 0    # next sample to emit
        self.carry = torch.zeros((self.S, self.C, -self.lead), dtype=torch.float32,
                                 device=self.device)  # global [t_emit + lead, t_end)
        self.stream = torch.cuda.Stream(device=self.device)
        # completion event of the last chunk's work (first: the carry's fill)
        self.done = torch.cuda.Event()
        self.done.record(torch.cuda.current_stream(self.device))
        self.results = []  # (g0, beam_max, argmax) device tensors, in order

    def bytes_per_chunk(self, n_samples):
        """Device bytes one chunk holds while in flight (record + traces + outputs)."""
        rec = n_samples + self.lag - self.lead
        elem = 4 if self._st == 0 else 2 * trace_copies(self._st)  # 16-bit: shifted copies
        return (self.S * self.C * rec * 4 + self.S * self.P * (rec + 1024 + self.lag) * elem
                + n_samples * 16)

    def _beamform(self, record, base, out_lo, out_hi):
        """Beamform record samples [out_lo, out_hi) of a record starting at
        global sample `base`.  Enqueued on the current stream."""
        T = int(record.shape[2])
        lpad, pitch = self.table.layout(T)
        st = self._st
        rows = self.S * self.P * trace_copies(st)
        elem = torch.float32 if st == 0 else (torch.bfloat16 if st == 1 else torch.float16)
        traces = torch.empty((rows, pitch), dtype=elem, device=self.device)
        scales = torch.ones(self.S, dtype=torch.float32, device=self.device)
        sp = _stream_ptr()
        check(self.lib.bp_prestack_dev(record.data_ptr(), self.alpha.data_ptr(), T, self.S,
                                       self.C, self.P, st, lpad, pitch, traces.data_ptr(),
                                       scales.data_ptr(), sp))
        n = out_hi - out_lo
        bm = torch.zeros(n, dtype=torch.float32, device=self.device)
        am = torch.zeros(n, dtype=torch.int32, device=self.device)
        keys = torch.empty(max(n, 1), dtype=torch.int64, device=self.device)
        r = Record()
        r.table = 0
        r.out_of_bounds = self.oob
        r.traces = traces.data_ptr()
        r.scales = scales.data_ptr()
        r.n_samples = T
        r.lpad = lpad
        r.pitch = pitch
        r.t_origin = base
        r.out0 = out_lo
        r.out1 = out_hi
        r.station_mask = None
        r.beam_max = bm.data_ptr()
        r.argmax = am.data_ptr()
        check(self.lib.bp_record_beamform_max_dev(self.table.handle, ct.byref(r), st,
                                                  keys.data_ptr(), sp))
        # keep the temporaries alive until the stream has used them
        for t in (traces, scales, keys, record):
            t.record_stream(torch.cuda.current_stream())
        return bm, am

    def _enter(self, stream):
        """Make `stream` (default: this network's own) wait for the previous
        chunk's work; returns it."""
        s = self.stream if stream is None else stream
        s.wait_event(self.done)
        # the carried halo was written on the previous chunk's stream
        self.carry.record_stream(s)
        return s

    def _leave(self, s):
        self.done = torch.cuda.Event()
        self.done.record(s)

    def push(self, chunk, stream=None, start_event=None):
        """Append an (S, C, L) chunk (numpy, host or device tensor); enqueue the
        work on `stream` (default: this network's own stream), after the
        previous chunk's work; `start_event` is recorded where the chunk's
        own work starts.  Returns the emitted (g0, beam_max, argmax) or None."""
        s = self._enter(stream)
        if start_event is not None:
            start_event.record(s)
        with torch.cuda.stream(s):
            if isinstance(chunk, np.ndarray):
                chunk = torch.from_numpy(np.ascontiguousarray(chunk, dtype=np.float32))
            chunk = chunk.to(self.device, dtype=torch.float32, non_blocking=True)
            L = int(chunk.shape[2])
            base = self.t_emit + self.lead
            record = torch.cat([self.carry, chunk], dim=2)  # global [base, t_end + L)
            self.t_end += L
            emit_to = self.t_end - self.lag
            out = None
            if emit_to > self.t_emit:
                bm, am = self._beamform(record, base, self.t_emit - base, emit_to - base)
                out = (self.t_emit, bm, am)
                self.results.append(out)
                self.t_emit = emit_to
            new_base = self.t_emit + self.lead
            self.carry = record[:, :, new_base - base:].contiguous()
        self._leave(s)
        return out

    def flush(self, stream=None):
        """End of the record: emit every remaining sample."""
        s = self._enter(stream)
        with torch.cuda.stream(s):
            base = self.t_emit + self.lead
            out = None
            if self.t_end > self.t_emit:
                bm, am = self._beamform(self.carry.contiguous(), base, self.t_emit - base,
                                        self.t_end - base)
                out = (self.t_emit, bm, am)
                self.results.append(out)
                self.t_emit = self.t_end
        self._leave(s)
        return out

    def synchronize(self):
        """Wait for every chunk enqueued so far."""
        self.stream.synchronize()
        self.done.synchronize()

    # ---- checkpoint / resume ------------------------------------------------
    def state(self):
        """Host snapshot of what the stream carries between chunks: the
        not-yet-emitted features (the max-delay halo) and the stream position.
        Results already emitted are the caller's (``collect``) and are not in
        the snapshot.  Synchronises the stream."""
        self.synchronize()
        info = self.table.info
        return {"carry": self.carry.cpu().numpy(), "t_end": self.t_end,
                "t_emit": self.t_emit, "lead": self.lead, "lag": self.lag,
                "n_sources": self.table.n_sources, "n_stations": self.S,
                "n_channels": self.C, "n_phases": self.P,
                "min_delay": info["min_delay"], "max_delay": info["max_delay"]}

    def restore(self, state):
        """Continue from a snapshot taken by ``state()`` (this object's table
        and weights must be the snapshot's network): later chunks give the
        results the uninterrupted stream would have given."""
        info = self.table.info
        for key, mine in (("n_sources", self.table.n_sources), ("n_stations", self.S),
                          ("n_channels", self.C), ("n_phases", self.P),
                          ("min_delay", info["min_delay"]), ("max_delay", info["max_delay"]),
                          ("lead", self.lead), ("lag", self.lag)):
            if int(state[key]) != int(mine):
                raise ValueError(f"snapshot of another network: {key} {state[key]} != {mine}")
        carry = np.asarray(state["carry"], dtype=np.float32)
        if carry.shape != (self.S, self.C, int(state["t_end"]) - int(state["t_emit"])
                           - self.lead):
            raise ValueError("snapshot carry does not match its stream position")
        self.synchronize()
        with torch.cuda.stream(self.stream):
            self.carry = torch.from_numpy(np.ascontiguousarray(carry)).to(self.device)
        self._leave(self.stream)
        self.t_end = int(state["t_end"])
        self.t_emit = int(state["t_emit"])
        self.results = []
        return self

    def save(self, path):
        """``state()`` written to an .npz file."""
        np.savez(path, **{k: np.asarray(v) for k, v in self.state().items()})

    def load(self, path):
        """``restore()`` from a file written by ``save()``."""
        with np.load(path) as z:
            return self.restore({k: z[k] for k in z.files})

    def collect(self):
        """All emitted results as numpy arrays (synchronises the stream)."""
        self.synchronize()
        if not self.results:
            return np.zeros(0, np.float32), np.zeros(0, np.int32)
        bm = torch.cat([r[1] for r in self.results]).cpu().numpy()
        am = torch.cat([r[2] for r in self.results]).cpu().numpy()
        return bm, am


_PRIORITY_STREAMS = {}  # device index -> [torch.cuda.Stream], highest priority first


def priority_streams(device):
    """This process's pool of CUDA streams of distinct priorities on
    `device`, highest first (priorities beyond the device's range are clamped
    by CUDA, so the pool stops at a repeat).  Shared by every scheduler: the
    caching allocator keeps its blocks per stream, so reused streams keep
    their warmed-up memory."""
    dev = torch.device(device)
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    pool = _PRIORITY_STREAMS.get(idx)
    if pool is None:
        pool, seen = [], set()
        for k in range(16):
            st = torch.cuda.Stream(device=idx, priority=-k)
            if st.priority in seen:
                break
            seen.add(st.priority)
            pool.append(st)
        pool.sort(key=lambda st: st.priority)
        _PRIORITY_STREAMS[idx] = pool
    return pool


class StreamScheduler:
    """Continuous batching of chunks from many networks.

    networks: dict name -> NetworkStream
    max_inflight: chunks admitted to the GPU at once
    memory_budget: device bytes the in-flight chunks may hold
    max_wait: seconds a chunk may wait for admission (None: no limit).  A
        chunk that waited longer ends its network's stream: skipping one
        chunk would break the carried halo, so that chunk and the network's
        later pending chunks are dropped (``timed_out``) and the network
        takes no more chunks.  ``cancel(name)`` ends a stream the same way on
        request; chunks already on the GPU complete.
    latency_budget: seconds from arrival to result that a chunk aims for; its
        deadline is arrival + budget (a dict gives per-network budgets).
        Pending chunks are admitted earliest deadline first; a network's own
        chunks keep their order (their deadlines increase with arrival).
    priorities: run admitted chunks on a pool of streams of graded priority
        (the device's range, highest first), the k-th oldest chunk in flight
        on the k-th highest; False: every chunk on its network's own stream.
    """

    def __init__(self, networks, max_inflight=8, memory_budget=150e9, max_wait=None,
                 latency_budget=0.05, priorities=True):
        self.networks = dict(networks)
        self.max_inflight = max_inflight
        self.memory_budget = memory_budget
        self.max_wait = max_wait
        self.latency_budget = latency_budget
        self._seq = itertools.count()
        self.closed = {}  # name -> "cancelled" or "timed out"
        self.peak_pending = 0  # deepest queue seen
        self.peak_inflight = 0
        self.peak_mem = 0  # most device bytes admitted at once
        self.cancelled = []  # (name, arrival) of chunks dropped by cancel()
        self.timed_out = []  # (name, arrival) of chunks dropped by max_wait
        self.pending = []  # heap of (deadline, seq, arrival, name, chunk)
        self.inflight = []  # (arrival, name, event, bytes, terms, admit, start event)
        self.mem_in_use = 0
        self.push_host_s = []  # host seconds spent enqueueing each admitted chunk
        self._free, self._free_t = 0, -1.0  # cached free device memory
        self.done = []  # (name, arrival, completion, terms)
        dev = next(iter(self.networks.values())).device
        self.device = dev
        self.prio_streams = priority_streams(dev) if priorities else []
        # device clock -> host clock
        torch.cuda.synchronize(dev)
        self._ev0 = torch.cuda.Event(enable_timing=True)
        self._ev0.record(torch.cuda.current_stream(dev))
        torch.cuda.synchronize(dev)
        self._host0 = time.perf_counter()

    def warm_up(self, chunks):
        """Push one chunk of every network (`chunks`: name -> chunk) through
        every stream this scheduler may use, so that the first requests find
        the memory they need already cached for each stream (a first
        allocation on a stream can wait for the work running on the GPU).
        The chunks continue each network's stream; synchronises."""
        targets = self.prio_streams or [None]
        for name, chunk in chunks.items():
            for s in targets:
                self.networks[name].push(chunk, stream=s)
        for net in self.networks.values():
            net.synchronize()

    def submit(self, name, chunk, arrival=None):
        if name not in self.networks:
            raise KeyError(f"unknown network {name!r}")
        if name in self.closed:
            raise ValueError(f"network {name!r} takes no more chunks ({self.closed[name]})")
        arrival = time.perf_counter() if arrival is None else arrival
        budget = (self.latency_budget.get(name, 0.05) if isinstance(self.latency_budget, dict)
                  else self.latency_budget)
        heapq.heappush(self.pending, (arrival + budget, next(self._seq), arrival, name, chunk))

    def _drop(self, name, reason, into):
        """End network `name`'s stream: its pending chunks leave the queue."""
        self.closed[name] = reason
        keep = []
        for item in sorted(self.pending):
            if item[3] == name:
                into.append((name, item[2]))
            else:
                keep.append(item)
        heapq.heapify(keep)
        self.pending = keep

    def cancel(self, name):
        """Stop network `name`: drop its chunks not yet admitted (returns how
        many); chunks already on the GPU complete."""
        before = len(self.cancelled)
        self._drop(name, "cancelled", self.cancelled)
        return len(self.cancelled) - before

    def _admit(self):
        while self.pending and len(self.inflight) < self.max_inflight:
            _deadline, _seq, arrival, name, chunk = self.pending[0]
            if self.max_wait is not None and time.perf_counter() - arrival > self.max_wait:
                self._drop(name, "timed out", self.timed_out)
                continue
            net = self.networks[name]
            need = net.bytes_per_chunk(int(chunk.shape[2]))
            if self.inflight and (self.mem_in_use + need > self.memory_budget or
                                  need > self._free_bytes()):
                break  # wait for memory to free up
            heapq.heappop(self.pending)
            admit = time.perf_counter()
            t_emit0 = net.t_emit
            stream = None
            if self.prio_streams:
                stream = self.prio_streams[min(len(self.inflight), len(self.prio_streams) - 1)]
            ev0 = torch.cuda.Event(enable_timing=True)
            net.push(chunk, stream=stream, start_event=ev0)
            self.push_host_s.append(time.perf_counter() - admit)
            terms = (net.t_emit - t_emit0) * net.table.n_sources * net.S * net.P
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(net.stream if stream is None else stream)
            self.inflight.append((arrival, name, ev, need, terms, admit, ev0))
            self.mem_in_use += need

    def _free_bytes(self):
        """The device's free memory, queried at most every 250 ms (the query
        takes driver locks that can stall the request loop)."""
        now = time.perf_counter()
        if now - self._free_t > 0.25:
            self._free, _ = torch.cuda.mem_get_info(self.device)
            self._free_t = now
        return self._free

    def _retire(self):
        keep = []
        for item in self.inflight:
            arrival, name, ev, need, terms, admit, ev_start = item
            if ev.query():
                done_t = self._host0 + self._ev0.elapsed_time(ev) / 1e3
                start_t = self._host0 + self._ev0.elapsed_time(ev_start) / 1e3
                self.done.append((name, arrival, done_t, terms, admit, start_t))
                self.mem_in_use -= need
            else:
                keep.append(item)
        self.inflight = keep

    def step(self):
        self.peak_pending = max(self.peak_pending, len(self.pending))
        self._retire()
        self._admit()
        self.peak_inflight = max(self.peak_inflight, len(self.inflight))
        self.peak_mem = max(self.peak_mem, self.mem_in_use)

    def drain(self):
        while self.pending or self.inflight:
            self.step()
            if self.inflight:
                time.sleep(1e-4)

    def stats(self):
        """Latency = device completion - arrival, split into the wait before
        admission (host), admission to the chunk's first device work, and its
        device time (first to last work of the chunk on its stream)."""
        if not self.done:
            return {}
        d = self.done
        lat = np.array([c - a for _, a, c, *_ in d])
        t0 = min(a for _, a, *_ in d)
        t1 = max(c for _, _, c, *_ in d)
        terms = sum(x[3] for x in d)
        pct = lambda v, q: float(np.percentile(v, q) * 1e3)  # noqa: E731
        wait = np.array([x[4] - x[1] for x in d])
        launch = np.array([x[5] - x[4] for x in d])
        device = np.array([x[2] - x[5] for x in d])
        per_net = {}
        for name in sorted({x[0] for x in d}):
            v = np.array([x[2] - x[1] for x in d if x[0] == name])
            dv = np.array([x[2] - x[5] for x in d if x[0] == name])
            per_net[name] = {"chunks": int(v.size), "p50_ms": pct(v, 50), "p99_ms": pct(v, 99),
                             "device_p50_ms": pct(dv, 50)}
        return {"chunks": len(d), "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                "max_ms": float(lat.max() * 1e3), "terms": terms,
                "terms_per_s": terms / max(t1 - t0, 1e-9), "span_s": t1 - t0,
                "wait_p50_ms": pct(wait, 50), "wait_p99_ms": pct(wait, 99),
                "admit_to_start_p50_ms": pct(launch, 50), "admit_to_start_p99_ms": pct(launch, 99),
                "device_p50_ms": pct(device, 50), "device_p99_ms": pct(device, 99),
                "enqueue_p50_ms": pct(np.array(self.push_host_s), 50),
                "enqueue_p99_ms": pct(np.array(self.push_host_s), 99),
                "peak_queue_depth": self.peak_pending, "peak_inflight": self.peak_inflight,
                "peak_device_bytes_admitted": self.peak_mem,
                "cancelled": len(self.cancelled), "timed_out": len(self.timed_out),
                "per_network": per_net}
