"""NetworkStream's carry arithmetic on the CPU: which samples each chunk
emits, which features it carries to the next, and the checkpoint of that
state.

The device call that beamforms a record (``_beamform``) is replaced by a
stand-in that, for every output sample g, combines the record's samples at
g + k for every delay k of the network's range, and asserts that each of
those samples that exists in the whole record is inside the record it was
given.  A sample emitted too early, or a halo carried too short, therefore
fails the assertion or changes the value; the stand-in run over the whole
record at once is the offline result.  That the device call itself gives
the reference's beams for a record starting at global sample ``base`` is
tests/test_gpu_stream.py.
"""
import numpy as np
import pytest
import torch

from beampower_b200.stream import NetworkStream


class FakeTable:
    def __init__(self, dmin, dmax):
        self.info = {"min_delay": dmin, "max_delay": dmax}
        self.n_sources = 1


def window_sum(rec, base, lo, hi, dmin, dmax, t_total):
    """Stand-in beam of samples [lo, hi) of `rec` (record coordinates; the
    record starts at global sample `base`)."""
    T = rec.shape[-1]
    out = np.zeros(hi - lo)
    for j in range(lo, hi):
        acc = 0.0
        for k in range(dmin, dmax + 1):
            g = base + j + k
            if g < 0 or g >= t_total:
                continue  # not in the whole record either
            idx = j + k
            assert 0 <= idx < T, f"sample {g} needed but not carried / not yet received"
            acc += rec[idx] * (k - dmin + 1)
        out[j - lo] = acc
    return out


class HostStream(NetworkStream):
    """NetworkStream with host tensors and the device call replaced."""

    def __init__(self, dmin, dmax, t_total, S=2, C=3, P=2):
        self.table = FakeTable(dmin, dmax)
        self.S, self.C, self.P = S, C, P
        self.device = "cpu"
        self.stream = None
        self.dmin, self.dmax, self.t_total = dmin, dmax, t_total
        self.lead, self.lag = min(0, dmin), max(0, dmax)
        self.t_end = self.t_emit = 0
        self.carry = torch.zeros((S, C, -self.lead), dtype=torch.float32)
        self.results = []

    def _enter(self, stream):
        return None

    def _leave(self, s):
        pass

    def synchronize(self):
        pass

    def _beamform(self, record, base, out_lo, out_hi):
        rec = record.double().sum(dim=(0, 1)).numpy()
        bm = window_sum(rec, base, out_lo, out_hi, self.dmin, self.dmax, self.t_total)
        return torch.from_numpy(bm), torch.arange(base + out_lo, base + out_hi)


def offline(F, dmin, dmax):
    rec = F.astype(np.float64).sum(axis=(0, 1))
    return window_sum(rec, 0, 0, rec.size, dmin, dmax, rec.size)


DELAYS = [(0, 50), (-30, 40), (-20, -5), (5, 5), (0, 0), (-7, 0), (3, 120)]


def _chunks(rng, T):
    cuts = [0]
    while cuts[-1] < T:
        step = int(rng.choice([0, 1, 3, 17, 64, 150, 400]))
        cuts.append(min(T, cuts[-1] + step))
    return list(zip(cuts[:-1], cuts[1:]))


@pytest.mark.parametrize("dmin,dmax", DELAYS)
@pytest.mark.parametrize("seed", range(3))
def test_streamed_equals_offline(dmin, dmax, seed):
    rng = np.random.default_rng(seed)
    T = int(rng.integers(200, 1200))
    F = rng.standard_normal((2, 3, T)).astype(np.float32)
    net = HostStream(dmin, dmax, T)
    for a, b in _chunks(rng, T):
        net.push(F[:, :, a:b])
        # never emits a sample whose last needed trace sample is still to come
        assert net.t_emit <= max(0, net.t_end - net.lag)
        # the carry is what the next chunk needs, and no more
        assert net.carry.shape[2] == net.t_end - net.t_emit - net.lead
    net.flush()
    bm, am = net.collect()
    assert np.array_equal(am, np.arange(T))  # each sample once, in order
    assert np.array_equal(bm, offline(F, dmin, dmax))


@pytest.mark.parametrize("dmin,dmax", [(-30, 40), (0, 50)])
def test_checkpoint_resume_on_host(dmin, dmax, tmp_path):
    rng = np.random.default_rng(11)
    T = 900
    F = rng.standard_normal((2, 3, T)).astype(np.float32)
    first = HostStream(dmin, dmax, T)
    for a, b in [(0, 100), (100, 130), (130, 400)]:
        first.push(F[:, :, a:b])
    bm0, am0 = first.collect()
    path = tmp_path / "stream.npz"
    first.save(path)
    second = HostStream(dmin, dmax, T).load(path)
    for a, b in [(400, 650), (650, 900)]:
        second.push(F[:, :, a:b])
    second.flush()
    bm1, am1 = second.collect()
    assert np.array_equal(np.concatenate([am0, am1]), np.arange(T))
    assert np.array_equal(np.concatenate([bm0, bm1]), offline(F, dmin, dmax))
    # a snapshot of another network is refused
    with pytest.raises(ValueError):
        HostStream(dmin - 1, dmax, T).load(path)
