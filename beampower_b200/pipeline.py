"""The reference tutorial end to end on the GPU: raw waveforms and travel
times in, detections out.

notebooks/3_beampower.ipynb runs, in order: the envelope feature of every
trace (:145-147), the conversion of travel times to sample delays (:394),
``beampower.beamform(..., reduce="max")`` (:463), the time-dependent
threshold (:588) and the peaks above it (:618-626).  ``detect_events`` runs
the same steps on the device, each with the tutorial's arguments, with no
host round trip between them.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import detection
from .tables import TravelTimeTable

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


@dataclass
class Events:
    """Detections: sample index, beam value and winning source of each event,
    plus the beam series and the threshold they were read from."""

    peaks: object
    heights: object
    sources: object
    beam_max: object
    beam_argmax: object
    threshold: object


def detect_events(waveforms, travel_times, sampling_rate, weights_phases, weights_sources,
                  window_duration_sec=7200.0, num_dev=8.0, threshold_type="rms", overlap=0.66,
                  min_detection_interval_sec=60.0, relative_delays=False, out_of_bounds="strict",
                  storage="fp32", white_noise=None, seed=0, clip_max=1e5, table=None):
    """Detections of the tutorial from raw data.

    waveforms: (S, C, T) raw traces; travel_times: (N, S, P) seconds (ignored
    when a resident ``table`` built from them is given); weights as in
    ``beamform``.  Window and distance in seconds, converted with
    ``int(seconds * sampling_rate)`` as the tutorial does.  Returns Events
    with CUDA tensors.
    """
    if torch is None:
        raise RuntimeError("torch is required for detect_events")
    if table is None:
        table = TravelTimeTable.from_travel_times(travel_times, sampling_rate, weights_sources,
                                                  relative=relative_delays)
    traces = table.traces_from_waveforms(waveforms, weights_phases, storage=storage,
                                         clip_max=clip_max)
    oob = 0 if out_of_bounds == "strict" else 1
    beam_max, beam_argmax = table.beamform_max(traces, oob)
    window = int(window_duration_sec * sampling_rate)
    thr = detection.time_dependent_threshold(beam_max, window, overlap=overlap,
                                             threshold_type=threshold_type, num_dev=num_dev,
                                             white_noise=white_noise, seed=seed)
    d = detection.detect(beam_max, beam_argmax, threshold=thr,
                         distance=int(min_detection_interval_sec * sampling_rate))
    return Events(peaks=d.peaks, heights=d.heights, sources=d.sources, beam_max=beam_max,
                  beam_argmax=beam_argmax, threshold=thr)
