"""The tutorial end to end on the GPU (``pipeline.detect_events``) against
the same steps composed on the CPU: the oracle beamformer, threshold and
peak finder applied to the GPU's own envelope features.  Everything after the
features is exact, so the events must be identical; the features themselves
are checked against the tutorial in test_gpu_features.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_detect_events_equals_composed_steps(cuda, oracle_lib):
    import torch
    from oracle import detection as odet
    from beampower_b200.features import waveform_features
    from beampower_b200.pipeline import detect_events
    from beampower_b200.synthetic import SMALL, make_workload
    wl = make_workload(SMALL)
    fs = 25.0
    D, W, A = wl["time_delays"], wl["weights_sources"], wl["weights_phases"]
    # raw traces whose envelope peaks at the events: noise plus wave packets
    rng = np.random.default_rng(8)
    F = wl["waveform_features"]
    raw = (rng.standard_normal(F.shape) * (1.0 + F)).astype(np.float32)
    travel_times = (D / fs).astype(np.float32)
    win_sec, gap_sec = 40.0, 4.0
    n_zero_guess = 6000
    noise = rng.standard_normal(n_zero_guess).astype(np.float32)
    ev = detect_events(raw, travel_times, fs, A, W, window_duration_sec=win_sec, num_dev=3.0,
                       min_detection_interval_sec=gap_sec, white_noise=noise)
    # the same steps on the CPU, from the GPU's features
    feats = waveform_features(raw)
    U = oracle_lib.prestack(feats, A)
    bm, am = oracle_lib.beamform_max(U, D, W, 0)
    assert np.array_equal(ev.beam_max.cpu().numpy().view(np.uint32), bm.view(np.uint32))
    assert np.array_equal(ev.beam_argmax.cpu().numpy(), am)
    thr = odet.time_dependent_threshold(bm, int(win_sec * fs), 0.66, "rms", 3.0, noise)
    assert np.array_equal(ev.threshold.cpu().numpy().view(np.uint32), thr.view(np.uint32))
    peaks = odet.detect(bm, thr, int(gap_sec * fs))
    assert peaks.size > 0
    assert np.array_equal(ev.peaks.cpu().numpy(), peaks)
    assert np.array_equal(ev.sources.cpu().numpy(), am[peaks])
    assert isinstance(ev.peaks, torch.Tensor)
