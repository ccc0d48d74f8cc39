"""Sources split over GPUs, one process per GPU (torch.distributed).

The reference beamforms with every visible GPU by giving each a block of
sources and merging the partial maxima on the host
(beampower/src/beamform.cu:227-276, 430-445).  Here each rank (one process
per GPU, NCCL over NVLink) builds the table of its contiguous block of
sources, beamforms it into packed (beam, source) keys, and one elementwise
max all-reduce of T int64 keys (8 T bytes) merges the ranks; every rank then
decodes the same (beam_max, argmax), equal bit for bit to the single-GPU
call.  Without an initialised process group the call runs on one GPU.
"""
from __future__ import annotations

import numpy as np

from .core import check, load_library

try:
    import torch
    import torch.distributed as dist
except ImportError:  # pragma: no cover
    torch = None
    dist = None


def shard_range(n_sources, rank, world):
    """[lo, hi) of this rank's contiguous block; blocks differ by at most one
    source and cover [0, n_sources) in rank order."""
    base, extra = divmod(int(n_sources), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def world_of(group=None):
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def merge_keys(shared_keys, group=None):
    """Elementwise max over ranks of keys in signed order (int64 tensor, in
    place).  Works on any backend: NCCL for device keys, gloo for host keys."""
    _rank, world = world_of(group)
    if world > 1:
        dist.all_reduce(shared_keys, op=dist.ReduceOp.MAX, group=group)
    return shared_keys


class _NoTraces:
    """Trace stand-in of an empty block: only the record length matters."""

    def __init__(self, n_samples):
        self.n_samples = n_samples


def decode_shared(shared_keys, device=None):
    """(beam_max, argmax) from merged keys in signed order (zeros / 0 where
    no source is a candidate)."""
    from .tables import _stream_ptr
    T = int(shared_keys.shape[0])
    dev = shared_keys.device if device is None else device
    bm = torch.zeros(T, dtype=torch.float32, device=dev)
    am = torch.zeros(T, dtype=torch.int32, device=dev)
    check(load_library("gpu").bp_keys_from_shared_dev(shared_keys.data_ptr(), T, bm.data_ptr(),
                                                      am.data_ptr(), _stream_ptr()))
    return bm, am


class ShardedTable:
    """This rank's block of a travel-time table.

    time_delays (N, S, P) and weights_sources (N, S): the whole grid (numpy
    or tensors); only rows [lo, hi) are copied to this rank's GPU.
    """

    def __init__(self, time_delays, weights_sources, group=None, device=None, rank=None,
                 world=None):
        from .tables import TravelTimeTable
        self.group = group
        self.rank, self.world = world_of(group)
        if rank is not None:  # an explicit block (several blocks on one GPU)
            self.rank, self.world = int(rank), int(world)
        n = int(time_delays.shape[0])
        self.n_sources = n
        self.lo, self.hi = shard_range(n, self.rank, self.world)
        self.lib = load_library("gpu")
        self.table = None
        if self.hi > self.lo:
            D = time_delays[self.lo:self.hi]
            W = weights_sources[self.lo:self.hi]
            if isinstance(D, np.ndarray):
                D, W = np.ascontiguousarray(D), np.ascontiguousarray(W)
            self.table = TravelTimeTable(D, W, device=device)
            self.device = self.table.device
        else:  # more ranks than sources: this block is empty
            self.device = torch.device(device) if device is not None else torch.device(
                "cuda", torch.cuda.current_device())

    def traces_from_features(self, waveform_features, weights_phases, storage="fp32"):
        if self.table is None:
            return _NoTraces(int(waveform_features.shape[-1]))
        return self.table.traces_from_features(waveform_features, weights_phases,
                                               storage=storage)

    def shared_keys(self, traces, out_of_bounds=0):
        """This block's keys, rebased to global source indexes and in signed
        order (int64 CUDA tensor of n_samples), ready for the max over ranks."""
        from .tables import _stream_ptr
        T = traces.n_samples
        keys = torch.zeros(max(T, 1), dtype=torch.int64, device=self.device)
        if self.table is not None:
            bm = torch.zeros(T, dtype=torch.float32, device=self.device)
            am = torch.zeros(T, dtype=torch.int32, device=self.device)
            self.table.beamform_max(traces, out_of_bounds, out=(bm, am, keys))
        check(self.lib.bp_keys_to_shared_dev(keys.data_ptr(), T, self.lo, _stream_ptr()))
        return keys[:T]

    def beamform_max(self, traces, out_of_bounds=0):
        """(beam_max, argmax) over all ranks' sources, on every rank (CUDA
        tensors; argmax holds global source indexes)."""
        keys = merge_keys(self.shared_keys(traces, out_of_bounds), self.group)
        return decode_shared(keys, self.device)

    def close(self):
        if self.table is not None:
            self.table.close()


def beamform_max_sharded(waveform_features, time_delays, weights_phases, weights_sources,
                         out_of_bounds="strict", storage="fp32", group=None):
    """``beamform(..., reduce='max')`` with the sources split over the ranks of
    ``group`` (every rank passes the same arguments and gets the result)."""
    st = ShardedTable(time_delays, weights_sources, group=group)
    traces = st.traces_from_features(waveform_features, weights_phases, storage=storage)
    bm, am = st.beamform_max(traces, 0 if out_of_bounds == "strict" else 1)
    st.close()
    return bm, am
