"""C-ABI argument checks of the detection, feature and travel-time entry
points, and the trace-copy count.  Every call here is rejected (or is empty)
before any CUDA work, so this runs without a GPU."""
import ctypes as ct

import pytest

INVALID = 1


@pytest.fixture(scope="module")
def lib(bplib):
    return bplib


def test_trace_copies(lib):
    assert lib.bp_trace_copies(0) == 1
    assert lib.bp_trace_copies(1) == 4 and lib.bp_trace_copies(2) == 4
    assert lib.bp_trace_copies(7) == -1


def test_threshold_rejects(lib):
    buf = ct.c_void_p(1)  # never dereferenced: every call below is rejected first
    # NULL series, NULL output
    assert lib.bp_threshold_dev(None, 100, 10, 0.66, 0, 8.0, None, 0, 0, buf, None) == INVALID
    assert lib.bp_threshold_dev(buf, 100, 10, 0.66, 0, 8.0, None, 0, 0, None, None) == INVALID
    # series not longer than the window, bad kind, window step below 1
    assert lib.bp_threshold_dev(buf, 100, 100, 0.66, 0, 8.0, None, 0, 0, buf, None) == INVALID
    assert lib.bp_threshold_dev(buf, 100, 10, 0.66, 2, 8.0, None, 0, 0, buf, None) == INVALID
    assert lib.bp_threshold_dev(buf, 100, 10, 0.95, 0, 8.0, None, 0, 0, buf, None) == INVALID
    assert lib.bp_threshold_dev(buf, 100, 0, 0.66, 0, 8.0, None, 0, 0, buf, None) == INVALID


def test_peaks_and_detect_reject(lib):
    buf = ct.c_void_p(1)
    n = ct.c_size_t(123)
    # 0 < distance < 1 (SciPy raises), too small a capacity, NULL count
    assert lib.bp_find_peaks_dev(buf, 100, 0.5, buf, 50, ct.byref(n), None) == INVALID
    assert n.value == 0
    assert lib.bp_find_peaks_dev(buf, 100, 3.0, buf, 49, ct.byref(n), None) == INVALID
    assert lib.bp_find_peaks_dev(buf, 100, 3.0, buf, 50, None, None) == INVALID
    assert lib.bp_detect_dev(buf, None, buf, 100, 0.5, buf, buf, None, 50, ct.byref(n),
                             None) == INVALID
    assert lib.bp_detect_dev(buf, None, None, 100, 2.0, buf, buf, None, 50, ct.byref(n),
                             None) == INVALID


def test_peak_options_reject(lib):
    """bp_find_peaks_opt_dev: SciPy's argument errors, before any CUDA work."""
    from beampower_b200.core import PeakOptions
    buf = ct.c_void_p(1)
    n = ct.c_size_t(123)

    def opts(**kw):
        o = PeakOptions()
        for name in ("height", "threshold", "prominence"):
            setattr(o, f"{name}_min", float("nan"))
            setattr(o, f"{name}_max", float("nan"))
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def call(o, cap=50, count=ct.byref(n)):
        return lib.bp_find_peaks_opt_dev(buf, 100, None if o is None else ct.byref(o), buf,
                                         None, None, None, cap, count, None)

    assert call(None) == INVALID                                   # no options
    assert call(opts(), count=None) == INVALID                     # no count
    assert call(opts(distance=0.5)) == INVALID and n.value == 0    # 0 < distance < 1
    assert call(opts(use_prominence=1, wlen=1.0)) == INVALID       # ceil(wlen) <= 1
    assert call(opts(), cap=49) == INVALID                         # capacity < n / 2
    assert lib.bp_find_peaks_opt_dev(None, 100, ct.byref(opts()), buf, None, None, None, 50,
                                     ct.byref(n), None) == INVALID  # NULL series


def test_features_and_ingest_reject_or_empty(lib):
    buf = ct.c_void_p(1)
    assert lib.bp_envelope_dev(None, 2, 10, 1e5, buf, None) == INVALID
    assert lib.bp_envelope_dev(buf, 2, 10, 1e5, None, None) == INVALID
    assert lib.bp_envelope_dev(None, 0, 10, 1e5, None, None) == 0  # nothing to do
    assert lib.bp_prestack_envelope_dev(None, buf, 10, 2, 3, 2, 1e5, 0, 0, 10, buf, None,
                                        None) == INVALID
    assert lib.bp_seconds_to_samples_dev(None, 1, 1, 25.0, 0.2, 0, buf, None) == INVALID
    assert lib.bp_seconds_to_samples_dev(None, 0, 5, 25.0, 0.2, 0, None, None) == 0
