"""Sources split into blocks on one GPU (the ranks' work done one after the
other, the max over ranks taken with torch): the merged (beam_max, argmax)
equal the single-GPU call bit for bit, strict and flexible, for 1 to 5
blocks, an empty block included; and a one-rank NCCL process group runs the
collective path."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("blocks", [1, 2, 3, 5])
@pytest.mark.parametrize("oob", [0, 1])
def test_blocks_merge_to_single_gpu_result(cuda, bplib, blocks, oob):
    import torch
    from beampower_b200.distributed import ShardedTable, decode_shared
    from beampower_b200.tables import TravelTimeTable
    from beampower_b200.synthetic import SMALL, make_workload
    wl = make_workload(SMALL)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    full = TravelTimeTable(D, W)
    bm, am = full.beamform_max(full.traces_from_features(F, A), oob)
    merged = None
    for r in range(blocks):
        st = ShardedTable(D, W, rank=r, world=blocks)
        k = st.shared_keys(st.traces_from_features(F, A), oob)
        merged = k.clone() if merged is None else torch.maximum(merged, k)
        st.close()
    gbm, gam = decode_shared(merged)
    torch.cuda.synchronize()
    assert np.array_equal(_bits(gbm.cpu().numpy()), _bits(bm.cpu().numpy()))
    assert np.array_equal(gam.cpu().numpy(), am.cpu().numpy())
    full.close()


def test_more_blocks_than_sources(cuda):
    import torch
    from beampower_b200.distributed import ShardedTable, decode_shared
    g = load_golden("tiny_all_zero_source")  # 33 sources
    bm_ref = g["beam_max_strict"]
    merged = None
    for r in range(40):  # seven blocks are empty
        st = ShardedTable(g["D"], g["W"], rank=r, world=40)
        k = st.shared_keys(st.traces_from_features(g["F"], g["A"]), 0)
        merged = k.clone() if merged is None else torch.maximum(merged, k)
        st.close()
    bm, am = decode_shared(merged)
    assert np.array_equal(_bits(bm.cpu().numpy()), _bits(bm_ref))
    assert np.array_equal(am.cpu().numpy(), g["argmax_strict"])


def test_one_rank_nccl_group(cuda):
    import os
    import socket
    import torch.distributed as dist
    from beampower_b200.distributed import beamform_max_sharded
    g = load_golden("random_p2")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        bm, am = beamform_max_sharded(g["F"], g["D"], g["A"], g["W"])
        assert np.array_equal(_bits(bm.cpu().numpy()), _bits(g["beam_max_strict"]))
        assert np.array_equal(am.cpu().numpy(), g["argmax_strict"])
    finally:
        dist.destroy_process_group()
