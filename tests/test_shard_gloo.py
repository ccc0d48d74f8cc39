"""The merge step of sources split over ranks, with the gloo backend on CPU
(world_size 2 and 3): each rank holds keys in signed order (what
bp_keys_to_shared_dev writes), the elementwise max over ranks must equal the
unsigned max of the original keys, and the source blocks must tile the grid.
The GPU side (rebase, decode, equality with the single-GPU call) is in
tests/test_gpu_shard.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

SIGN = np.uint64(1 << 63)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_keys(rank, n):
    """Keys of one rank: random beams packed as ordered(beam) << 32 |
    (0xFFFFFFFF - source), some samples without a candidate (key 0)."""
    rng = np.random.default_rng(100 + rank)
    hi = rng.integers(1, 2**32, size=n, dtype=np.uint64)
    lo = rng.integers(0, 2**32, size=n, dtype=np.uint64)
    keys = (hi << np.uint64(32)) | lo
    keys[rng.random(n) < 0.2] = 0
    keys[:3] = 0  # a few samples where no rank has a candidate
    return keys


def _worker(rank, world, port, n, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from beampower_b200 import distributed as bd
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert bd.world_of() == (rank, world)
        shared = torch.from_numpy((_rank_keys(rank, n) ^ SIGN).view(np.int64).copy())
        bd.merge_keys(shared)
        out.put((rank, shared.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_merge_over_ranks_gloo(world):
    n = 5000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.max(np.stack([_rank_keys(r, n) for r in range(world)]), axis=0)
    for r in range(world):
        got = res[r].view(np.uint64) ^ SIGN
        assert np.array_equal(got, want)
    assert np.all(want[:3] == 0)


@pytest.mark.parametrize("n,world", [(0, 2), (1, 3), (7, 8), (400000, 8), (1001, 4)])
def test_shard_ranges_tile_the_grid(n, world):
    from beampower_b200.distributed import shard_range
    spans = [shard_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1
