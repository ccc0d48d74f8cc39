"""Multi-process replica measurement with the gloo backend on CPU
(world_size 2): barrier, max over ranks, whole-job rate."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from beampower_b200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert replicas.world() == (rank, world, rank)
        replicas.barrier()
        elapsed = 1.0 + rank  # rank 1 is the slow one
        rate, slowest = replicas.whole_job_rate(100.0, elapsed)
        out.put((rank, rate, slowest, replicas.max_over_ranks(-rank)))
        replicas.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, slowest, mx in res:
        assert slowest == 2.0            # the max over ranks
        assert rate == pytest.approx(2 * 100.0 / 2.0)  # all ranks' work / slowest time
        assert mx == 0.0


def test_single_process_identity():
    from beampower_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.whole_job_rate(10.0, 2.0) == (5.0, 2.0)
