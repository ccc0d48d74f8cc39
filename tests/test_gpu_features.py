"""Envelope features on the GPU against the tutorial fixtures and the oracle.

The FFTs are float32 (cuFFT here, SciPy's pocketfft in the tutorial), so the
comparison has a tolerance.  Both envelopes carry rounding errors of up to
delta * max|envelope|, delta of order eps * log2(T); the median and the MAD
(median absolute deviation) inherit errors of the same size.  The feature
f = (envelope - median) / MAD therefore differs, to first order, by at most

    |gpu - tutorial| <= delta * kappa * (2 + |tutorial|),  kappa = max|envelope| / MAD

with delta = 1e-5 (above 4 * eps * log2(T) up to T = 10^7) and kappa from the
tutorial's own envelope.  kappa is the trace's conditioning: about 10^2 for
the seismic-like traces, 5e5 for the spike trace, whose MAD is at the FFT
rounding level of the spike (there the check is mostly that the clip at 1e5
holds).
"""

import numpy as np
import pytest

from test_features_oracle import G, NAMES

pytestmark = pytest.mark.gpu


def _bound(raw, ref):
    med = np.median(raw)
    mad = np.median(np.abs(raw - med))
    mad = 1.0 if mad == 0 else mad
    kappa = float(np.max(np.abs(raw), initial=0.0)) / mad
    return 1e-5 * kappa * (2.0 + np.abs(ref.astype(np.float64)))


@pytest.mark.parametrize("name", NAMES)
def test_envelope_matches_tutorial(cuda, name):
    from beampower_b200.features import envelope
    x, ref, raw = G[f"x_{name}"], G[f"feature_{name}"], G[f"raw_{name}"]
    got = envelope(x)
    assert got.shape == x.shape and got.dtype == np.float32
    err = np.abs(got.astype(np.float64) - ref)
    assert np.all(err <= _bound(raw, ref)), (name, float(err.max()))
    assert np.all(got <= np.float32(1e5))


def test_rows_and_tensors(cuda):
    import torch
    from beampower_b200.features import envelope
    x = np.stack([G["x_even_1000"], -G["x_even_1000"], 3 * G["x_even_1000"]])
    got = envelope(torch.from_numpy(x).to(cuda))
    assert isinstance(got, torch.Tensor) and got.is_cuda
    one = envelope(G["x_even_1000"])
    g = got.cpu().numpy()
    # the three rows have one envelope up to sign and scale: one feature
    bound = _bound(G["raw_even_1000"], G["feature_even_1000"])
    for r in range(3):
        assert np.all(np.abs(g[r].astype(np.float64) - one) <= 2 * bound), r


def test_network_against_oracle(cuda):
    """20 stations x 3 channels x 180,000 samples of seismic-like noise with
    events, against the CPU oracle, row by row with the bound above."""
    from oracle import features as ofeat
    from beampower_b200.features import waveform_features
    rng = np.random.default_rng(3)
    S, C, T = 20, 3, 180000
    w = rng.standard_normal((S, C, T)).astype(np.float32)
    for s in range(S):
        t0 = rng.integers(1000, T - 1000, size=5)
        for t in t0:
            w[s, :, t:t + 200] += (rng.uniform(5, 20) * np.sin(0.5 * np.arange(200))
                                   ).astype(np.float32)
    got = waveform_features(w)
    from scipy import signal
    for s in range(0, S, 4):
        for c in range(C):
            ref = ofeat.envelope(w[s, c])
            raw = np.abs(signal.hilbert(w[s, c]))
            err = np.abs(got[s, c].astype(np.float64) - ref)
            assert np.all(err <= _bound(raw, ref)), (s, c, float(err.max()))


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_traces_from_waveforms_equals_two_step_path(cuda, storage):
    """Raw waveforms -> trace rows in one call gives the very trace rows of
    envelope features followed by the prestack, so the beams are identical."""
    import torch
    from beampower_b200.features import waveform_features
    from beampower_b200.tables import TravelTimeTable
    rng = np.random.default_rng(4)
    S, C, P, T, N = 8, 3, 2, 5000, 500
    w = rng.standard_normal((S, C, T)).astype(np.float32)
    A = rng.uniform(0, 1, size=(S, C, P)).astype(np.float32)
    D = rng.integers(0, 300, size=(N, S, P)).astype(np.int32)
    W = rng.uniform(0.5, 1.5, size=(N, S)).astype(np.float32)
    table = TravelTimeTable(D, W)
    a = table.traces_from_waveforms(w, A, storage=storage)
    b = table.traces_from_features(waveform_features(w), A, storage=storage)
    torch.cuda.synchronize()
    view = torch.int32 if storage == "fp32" else torch.int16
    assert torch.equal(a.buf.view(view), b.buf.view(view))
    assert torch.equal(a.scales, b.scales)
    bm_a, am_a = table.beamform_max(a, 0)
    bm_b, am_b = table.beamform_max(b, 0)
    assert torch.equal(bm_a, bm_b) and torch.equal(am_a, am_b)
    table.close()


def test_edge_shapes(cuda):
    from beampower_b200.features import envelope
    assert envelope(np.zeros((3, 0), np.float32)).shape == (3, 0)
    assert np.array_equal(envelope(np.array([5.0], np.float32)), np.zeros(1, np.float32))
    z = envelope(np.zeros(64, np.float32))
    assert np.array_equal(z, np.zeros(64, np.float32))
