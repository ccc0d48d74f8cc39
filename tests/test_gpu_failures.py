"""Failure handling without faulting a GPU: a wait that can never complete
ends with an error status; malformed requests are refused before any
launch; the stream scheduler holds chunks back when the memory budget is
full instead of over-committing."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout(cuda, bplib):
    import torch
    from beampower_b200.tables import _stream_ptr
    st = ct.c_int(-1)
    assert bplib.bp_debug_wait_timeout(2_000_000, _stream_ptr(), ct.byref(st)) == 0
    assert st.value == 1  # wait timeout bit
    # the context is still usable afterwards
    x = torch.arange(10, device="cuda").sum().item()
    assert x == 45


def test_malformed_requests_refused(cuda):
    import beampower_b200 as bp
    from beampower_b200.core import BeampowerError
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(0)
    D = rng.integers(0, 50, size=(100, 4, 2)).astype(np.int32)
    W = np.ones((100, 4), np.float32)
    with pytest.raises(ValueError):
        TravelTimeTable(D, W[:, :3])  # shape mismatch
    table = TravelTimeTable(D, W)
    with pytest.raises(ValueError):
        table.traces_from_features(np.ones((5, 3, 100), np.float32),
                                   np.ones((5, 3, 2), np.float32))
    lib = bp.load_library("gpu")
    # layout too small for the table: refused with a message, no launch
    import torch
    tr = table.traces_from_features(np.ones((4, 3, 100), np.float32), np.ones((4, 3, 2),
                                                                             np.float32))
    keys = torch.empty(100, dtype=torch.int64, device="cuda")
    bm = torch.zeros(100, device="cuda")
    am = torch.zeros(100, dtype=torch.int32, device="cuda")
    from beampower_b200.tables import _stream_ptr
    rc = lib.bp_beamform_max_dev(table.handle, tr.buf.data_ptr(), 0, None, 100, 0, 64, 0,
                                 keys.data_ptr(), bm.data_ptr(), am.data_ptr(), _stream_ptr())
    assert rc == 1 and b"layout" in lib.bp_last_error()
    with pytest.raises(BeampowerError):
        from beampower_b200.core import check
        check(rc)
    table.close()


def test_scheduler_respects_memory_budget(cuda):
    """With a budget below two chunks, one chunk at a time is in flight; the
    queue drains and every chunk completes."""
    from beampower_b200.stream import NetworkStream, StreamScheduler
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(1)
    S, C, P, N = 6, 3, 2, 400
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, 100, size=(N, S, P)).astype(np.int32)
    W = np.ones((N, S), np.float32)
    ns = NetworkStream(TravelTimeTable(D, W), A, storage="fp32")
    budget = int(1.5 * ns.bytes_per_chunk(500))
    sched = StreamScheduler({"n": ns}, max_inflight=8, memory_budget=budget)
    peak = 0
    for _ in range(6):
        sched.submit("n", np.abs(rng.standard_normal((S, C, 500))).astype(np.float32))
    while sched.pending or sched.inflight:
        sched.step()
        peak = max(peak, len(sched.inflight))
    assert peak == 1 and len(sched.done) == 6
    st = sched.stats()
    assert st["peak_inflight"] == 1 and st["peak_queue_depth"] >= 5
    assert 0 < st["peak_device_bytes_admitted"] <= budget


def _two_networks(rng):
    from beampower_b200.stream import NetworkStream
    from beampower_b200.tables import TravelTimeTable
    S, C, P, N = 6, 3, 2, 300
    nets, data = {}, {}
    for name in ("a", "b"):
        A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
        D = rng.integers(0, 80, size=(N, S, P)).astype(np.int32)
        W = np.ones((N, S), np.float32)
        nets[name] = NetworkStream(TravelTimeTable(D, W), A, storage="fp32")
        data[name] = (A, D, W, np.abs(rng.standard_normal((S, C, 1500))).astype(np.float32))
    return nets, data


def test_cancelled_stream(cuda, oracle_lib):
    """Cancelling network b drops its queued chunks and refuses new ones;
    network a streams on and still equals its offline call."""
    from beampower_b200.stream import StreamScheduler
    nets, data = _two_networks(np.random.default_rng(2))
    sched = StreamScheduler(nets, max_inflight=2)
    for i in range(3):
        for name in ("a", "b"):
            sched.submit(name, data[name][3][:, :, i * 500:(i + 1) * 500])
    assert sched.cancel("b") == 3
    with pytest.raises(ValueError):
        sched.submit("b", data["b"][3][:, :, :500])
    sched.drain()
    assert [x[0] for x in sched.done] == ["a"] * 3 and len(sched.cancelled) == 3
    nets["a"].flush()
    bm, am = nets["a"].collect()
    A, D, W, F = data["a"]
    obm, oam = oracle_lib.beamform_max(oracle_lib.prestack(F, A), D, W, 0)
    assert np.array_equal(bm.view(np.uint32), obm.view(np.uint32)) and np.array_equal(am, oam)


def test_queue_timeout_ends_that_stream(cuda):
    """A chunk that waited past max_wait ends its network's stream (its later
    queued chunks are dropped with it); the other network is served."""
    import time
    from beampower_b200.stream import StreamScheduler
    nets, data = _two_networks(np.random.default_rng(3))
    sched = StreamScheduler(nets, max_inflight=2, max_wait=1.0)
    now = time.perf_counter()
    for i in range(2):
        sched.submit("b", data["b"][3][:, :, i * 500:(i + 1) * 500], arrival=now - 10.0)
        sched.submit("a", data["a"][3][:, :, i * 500:(i + 1) * 500])
    sched.drain()
    assert len(sched.timed_out) == 2 and sched.closed == {"b": "timed out"}
    assert [x[0] for x in sched.done] == ["a", "a"]
    with pytest.raises(ValueError):
        sched.submit("b", data["b"][3][:, :, :500])
