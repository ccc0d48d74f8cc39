"""The stream scheduler's request loop on the CPU: admission order (earliest
deadline first), the in-flight and memory limits, the wait limit and
cancel, and the latency statistics.

The networks are fakes that record the order in which chunks are pushed, and
CUDA events are replaced by host objects whose completion and device time the
test sets, so that only the scheduler's own host logic runs.  Its GPU
behaviour (results identical alone and in the mix, deadline order on real
streams) is covered by tests/test_gpu_stream.py.
"""
import numpy as np
import pytest
import torch

from beampower_b200.stream import StreamScheduler


class FakeEvent:
    """Host stand-in for torch.cuda.Event: `t` is its device time (seconds),
    `done` whether the device has passed it."""

    def __init__(self, enable_timing=False):
        self.t = None
        self.done = False

    def record(self, stream=None):
        if self.t is None:
            self.t = 0.0

    def query(self):
        return self.done

    def elapsed_time(self, other):
        return (other.t - self.t) * 1e3


class FakeTable:
    def __init__(self, n_sources):
        self.n_sources = n_sources


class FakeNet:
    """A network whose chunk of L samples holds L * 1000 device bytes."""

    def __init__(self, name, log, n_sources=10, S=3, P=2):
        self.name, self.log = name, log
        self.device = "cpu"
        self.table = FakeTable(n_sources)
        self.S, self.P = S, P
        self.stream = object()
        self.t_emit = 0

    def bytes_per_chunk(self, n_samples):
        return n_samples * 1000

    def push(self, chunk, stream=None, start_event=None):
        if start_event is not None:
            start_event.record(stream)
        self.t_emit += int(chunk.shape[2])
        self.log.append((self.name, int(chunk[0, 0, 0])))

    def synchronize(self):
        pass


@pytest.fixture
def fake_cuda(monkeypatch):
    free = {"bytes": 1 << 40}
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a, **k: (free["bytes"], 1 << 40))
    return free


def chunk(tag, n_samples=4):
    """An (S, C, L) chunk whose first value tags it in the push log."""
    c = np.zeros((3, 1, n_samples), dtype=np.float32)
    c[0, 0, 0] = tag
    return c


def make(names, **kw):
    log = []
    nets = {n: FakeNet(n, log) for n in names}
    return StreamScheduler(nets, priorities=False, **kw), log


def complete(sched, k=None, t=1.0):
    """Mark the first k in-flight chunks (all by default) done at device time t."""
    for item in sched.inflight[:k]:
        item[2].done = True
        item[2].t = t
        item[6].t = min(item[6].t, t)


def test_earliest_deadline_first(fake_cuda):
    sched, log = make(["a", "b"], max_inflight=1, latency_budget={"a": 0.2, "b": 0.05})
    sched.submit("a", chunk(1), arrival=0.00)   # deadline 0.20
    sched.submit("b", chunk(2), arrival=0.10)   # deadline 0.15
    sched.submit("a", chunk(3), arrival=0.05)   # deadline 0.25
    sched.step()
    assert log == [("b", 2)]
    complete(sched)
    sched.step()
    complete(sched)
    sched.step()
    assert log == [("b", 2), ("a", 1), ("a", 3)]


def test_one_networks_chunks_keep_their_order(fake_cuda):
    sched, log = make(["a"], max_inflight=8, latency_budget=0.05)
    for k in range(5):
        sched.submit("a", chunk(k), arrival=1.0)  # equal arrivals: submission order
    sched.step()
    assert log == [("a", k) for k in range(5)]


def test_inflight_limit(fake_cuda):
    sched, log = make(["a", "b"], max_inflight=2)
    for k in range(3):
        sched.submit("a" if k % 2 == 0 else "b", chunk(k), arrival=float(k))
    sched.step()
    assert len(sched.inflight) == 2 and len(sched.pending) == 1
    complete(sched, 1)
    sched.step()
    assert [x[0] for x in log] == ["a", "b", "a"]
    assert sched.peak_inflight == 2


def test_memory_budget_holds_the_queue_head(fake_cuda):
    # 3,000-byte chunks against a 5,000-byte budget: one at a time; a small
    # chunk with a later deadline does not pass the waiting head
    sched, log = make(["a", "b"], max_inflight=8, memory_budget=5000)
    sched.submit("a", chunk(1, 3), arrival=0.0)
    sched.submit("b", chunk(2, 3), arrival=0.1)
    sched.submit("a", chunk(3, 1), arrival=0.2)
    sched.step()
    assert log == [("a", 1)] and sched.mem_in_use == 3000
    sched.step()
    assert log == [("a", 1)]
    complete(sched)
    sched.step()
    assert log == [("a", 1), ("b", 2), ("a", 3)]
    assert sched.mem_in_use == 4000 and sched.peak_mem == 4000


def test_chunk_larger_than_budget_runs_alone(fake_cuda):
    sched, log = make(["a"], max_inflight=8, memory_budget=1000)
    sched.submit("a", chunk(1, 5), arrival=0.0)
    sched.submit("a", chunk(2, 5), arrival=0.1)
    sched.step()
    assert log == [("a", 1)]
    complete(sched)
    sched.step()
    assert log == [("a", 1), ("a", 2)]


def test_free_device_memory_limits_admission(fake_cuda):
    fake_cuda["bytes"] = 5000
    sched, log = make(["a"], max_inflight=8)
    sched.submit("a", chunk(1, 4), arrival=0.0)
    sched.submit("a", chunk(2, 6), arrival=0.1)
    sched.step()
    assert log == [("a", 1)]  # 6,000 bytes > 5,000 free while one chunk runs


def test_wait_limit_ends_the_late_stream_only(fake_cuda):
    import time
    sched, log = make(["a", "b"], max_inflight=8, max_wait=0.5)
    now = time.perf_counter()
    sched.submit("a", chunk(1), arrival=now - 2.0)   # waited too long
    sched.submit("a", chunk(2), arrival=now)
    sched.submit("b", chunk(3), arrival=now)
    sched.step()
    assert log == [("b", 3)]
    assert sorted(a for _, a in sched.timed_out) == [now - 2.0, now]
    assert sched.closed == {"a": "timed out"}
    with pytest.raises(ValueError):
        sched.submit("a", chunk(4))


def test_cancel_drops_pending_chunks_only(fake_cuda):
    sched, log = make(["a", "b"], max_inflight=1)
    sched.submit("a", chunk(1), arrival=0.0)
    sched.submit("a", chunk(2), arrival=0.1)
    sched.submit("b", chunk(3), arrival=0.2)
    sched.step()
    assert sched.cancel("a") == 1
    assert len(sched.inflight) == 1  # the admitted chunk completes
    complete(sched)
    sched.step()
    assert log == [("a", 1), ("b", 3)]
    with pytest.raises(ValueError):
        sched.submit("a", chunk(5))
    with pytest.raises(KeyError):
        sched.submit("c", chunk(6))


def test_latency_statistics(fake_cuda):
    sched, log = make(["a", "b"], max_inflight=8)
    host0 = sched._host0
    sched.submit("a", chunk(1, 4), arrival=host0 + 0.000)
    sched.submit("b", chunk(2, 4), arrival=host0 + 0.010)
    sched.step()
    # device completions at 30 ms and 50 ms after the scheduler's time origin
    a_item, b_item = sched.inflight
    a_item[2].done, a_item[2].t = True, 0.030
    b_item[2].done, b_item[2].t = True, 0.050
    sched.step()
    st = sched.stats()
    assert st["chunks"] == 2
    assert st["per_network"]["a"]["p50_ms"] == pytest.approx(30.0)
    assert st["per_network"]["b"]["p50_ms"] == pytest.approx(40.0)
    assert st["max_ms"] == pytest.approx(40.0)
    # terms: samples emitted x sources x stations x phases
    assert st["terms"] == 2 * 4 * 10 * 3 * 2
    assert sched.mem_in_use == 0 and not sched.inflight
