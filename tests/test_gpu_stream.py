"""Stream scheduler: chunked, carried-over streaming equals one offline call
on the concatenated record (FP32: bit for bit, both rules, negative delays
included); continuous batching over several networks gives every network the
same result alone and in the mix."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHUNKS = [700, 333, 1500, 120, 900, 1447]


def bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return np.where(np.isnan(a), np.uint32(0x7FC00000), a.view(np.uint32))


def _net(seed, N=600, S=8, C=3, P=2, dlo=0, dhi=250):
    rng = np.random.default_rng(seed)
    A = rng.uniform(0.2, 1.2, size=(S, C, P)).astype(np.float32)
    D = rng.integers(dlo, dhi + 1, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.5, 1.5, size=(N, S)).astype(np.float32)
    W[rng.random(W.shape) < 0.15] = 0.0
    F = np.abs(rng.standard_normal((S, C, sum(CHUNKS)))).astype(np.float32)
    return A, D, W, F


def _stream(A, D, W, F, oob, storage="fp32"):
    from beampower_b200.stream import NetworkStream
    from beampower_b200.tables import TravelTimeTable
    ns = NetworkStream(TravelTimeTable(D, W), A, out_of_bounds=oob, storage=storage)
    t = 0
    for L in CHUNKS:
        ns.push(F[:, :, t:t + L])
        t += L
    ns.flush()
    return ns.collect()


@pytest.mark.parametrize("oob", ["strict", "flexible"])
@pytest.mark.parametrize("dlo", [0, -90])
def test_stream_equals_offline(cuda, oracle_lib, oob, dlo):
    A, D, W, F = _net(7 + abs(dlo), dlo=dlo)
    bm, am = _stream(A, D, W, F, oob)
    obm, oam = oracle_lib.beamform_max(oracle_lib.prestack(F, A), D, W,
                                       0 if oob == "strict" else 1)
    assert bm.shape == obm.shape
    assert np.array_equal(bits(bm), bits(obm))
    assert np.array_equal(am, oam)


def test_stream_16bit_within_tolerance(cuda, orc):
    """16-bit streaming: each chunk is scaled on its own record, so results
    match the float64 offline beams to the storage tolerance (FP16 1e-3)."""
    A, D, W, F = _net(11)
    bm, am = _stream(A, D, W, F, "strict", storage="fp16")
    beam64, valid = orc.fp64_beams(orc.fp64_prestack(F, A), D, W, 0)
    b = np.where(valid, beam64, -np.inf)
    top = b.max(axis=0)
    has = np.isfinite(top)
    rel = np.abs(bm[has] - top[has]) / np.abs(top[has])
    assert rel.max() <= 1e-3


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_scheduler_mix_equals_alone(cuda, storage):
    """Two networks' chunks interleaved through the continuous-batching
    scheduler (3 slots): each network's output equals its output alone (bit
    for bit: a chunk's arithmetic does not depend on what runs beside it)."""
    from beampower_b200.stream import NetworkStream, StreamScheduler
    from beampower_b200.tables import TravelTimeTable
    nets = {"a": _net(21, N=900, S=8), "b": _net(22, N=300, S=5, dhi=120)}
    alone = {k: _stream(*v, "strict", storage=storage) for k, v in nets.items()}
    streams = {k: NetworkStream(TravelTimeTable(v[1], v[2]), v[0], "strict", storage=storage,
                                 name=k)
               for k, v in nets.items()}
    sched = StreamScheduler(streams, max_inflight=3, memory_budget=2e9)
    offs = {k: 0 for k in nets}
    for L in CHUNKS:
        for k, v in nets.items():
            F = v[3]
            sched.submit(k, F[:, :, offs[k]:offs[k] + L])
            offs[k] += L
        sched.step()
    sched.drain()
    for k, ns in streams.items():
        ns.flush()
        bm, am = ns.collect()
        assert np.array_equal(bits(bm), bits(alone[k][0])), k
        assert np.array_equal(am, alone[k][1]), k
    st = sched.stats()
    assert st["chunks"] == 2 * len(CHUNKS) and st["p99_ms"] >= st["p50_ms"] >= 0


@pytest.mark.parametrize("oob,dlo", [("strict", 0), ("flexible", -90)])
@pytest.mark.parametrize("cut", [1, 3, 5])
def test_checkpoint_and_resume_equals_offline(cuda, oracle_lib, tmp_path, oob, dlo, cut):
    """Stream the first `cut` chunks, save the stream's state to a file,
    resume it in a fresh NetworkStream (new table object, as another process
    would build it), stream the rest: the two parts together equal one
    offline call bit for bit."""
    from beampower_b200.stream import NetworkStream
    from beampower_b200.tables import TravelTimeTable
    A, D, W, F = _net(30 + cut + abs(dlo), dlo=dlo)
    first = NetworkStream(TravelTimeTable(D, W), A, out_of_bounds=oob, storage="fp32")
    t = 0
    for L in CHUNKS[:cut]:
        first.push(F[:, :, t:t + L])
        t += L
    bm1, am1 = first.collect()
    path = tmp_path / "stream_state.npz"
    first.save(path)
    second = NetworkStream(TravelTimeTable(D, W), A, out_of_bounds=oob,
                           storage="fp32").load(path)
    for L in CHUNKS[cut:]:
        second.push(F[:, :, t:t + L])
        t += L
    second.flush()
    bm2, am2 = second.collect()
    bm, am = np.concatenate([bm1, bm2]), np.concatenate([am1, am2])
    obm, oam = oracle_lib.beamform_max(oracle_lib.prestack(F, A), D, W,
                                       0 if oob == "strict" else 1)
    assert np.array_equal(bits(bm), bits(obm)) and np.array_equal(am, oam)


def test_restore_rejects_another_network(cuda):
    from beampower_b200.stream import NetworkStream
    from beampower_b200.tables import TravelTimeTable
    A, D, W, F = _net(41)
    a = NetworkStream(TravelTimeTable(D, W), A, storage="fp32")
    a.push(F[:, :, :700])
    st = a.state()
    A2, D2, W2, _ = _net(42, N=500)
    with pytest.raises(ValueError):
        NetworkStream(TravelTimeTable(D2, W2), A2, storage="fp32").restore(st)


def test_scheduler_earliest_deadline_first(cuda):
    """Admission order is earliest deadline first (arrival + the network's
    latency budget) while each network's chunks stay in order; the priority
    pool holds streams of distinct, increasing priority values (highest
    first); results equal each network alone."""
    from beampower_b200.stream import NetworkStream, StreamScheduler
    from beampower_b200.tables import TravelTimeTable
    nets = {"a": _net(31, N=400, S=6), "b": _net(32, N=200, S=5, dhi=120)}
    alone = {k: _stream(*v, "strict", storage="fp16") for k, v in nets.items()}
    streams = {k: NetworkStream(TravelTimeTable(v[1], v[2]), v[0], "strict", name=k)
               for k, v in nets.items()}
    sched = StreamScheduler(streams, max_inflight=1, latency_budget={"a": 1.0, "b": 0.01})
    prios = [s.priority for s in sched.prio_streams]
    assert prios and prios == sorted(set(prios))
    offs = {k: 0 for k in nets}
    t0 = 1000.0
    for i, L in enumerate(CHUNKS):
        for k, v in nets.items():
            sched.submit(k, v[3][:, :, offs[k]:offs[k] + L], arrival=t0 + 0.001 * i)
            offs[k] += L
    sched.drain()
    # one chunk in flight at a time: completion order is admission order;
    # every chunk of b (deadline arrival + 10 ms) comes before a's (+ 1 s)
    order = [x[0] for x in sched.done]
    assert order == ["b"] * len(CHUNKS) + ["a"] * len(CHUNKS)
    for k, ns in streams.items():
        ns.flush()
        bm, am = ns.collect()
        assert np.array_equal(bits(bm), bits(alone[k][0])), k
        assert np.array_equal(am, alone[k][1]), k
