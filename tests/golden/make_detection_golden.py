"""Generate tests/golden/detection_*.npz from the reference tutorial itself.

The detection step of the tutorial (notebooks/3_beampower.ipynb:497-579,
``time_dependent_threshold``, and :618-626, find_peaks with a minimum
distance followed by the threshold test) lives in a notebook, not in the
package.  This script reads the notebook from the reference checkout, runs
the cell that defines ``time_dependent_threshold`` in a fresh namespace,
and calls it and ``scipy.signal.find_peaks`` on seeded series.  The white
noise the function draws for zero samples comes from NumPy's global
generator; the script seeds it before each call and stores the same draws,
so the fixtures hold every input the GPU path needs.

    python tests/golden/make_detection_golden.py [reference checkout]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
from scipy import signal

HERE = os.path.dirname(os.path.abspath(__file__))
NOTEBOOK = "notebooks/3_beampower.ipynb"


def load_threshold_function(ref_root):
    nb = json.load(open(os.path.join(ref_root, NOTEBOOK)))
    for cell in nb["cells"]:
        src = "".join(cell["source"])
        if cell["cell_type"] == "code" and "def time_dependent_threshold" in src:
            ns = {"np": np}
            exec(compile(src, NOTEBOOK, "exec"), ns)
            return ns["time_dependent_threshold"]
    raise RuntimeError("time_dependent_threshold not found in " + NOTEBOOK)


def beam_like(rng, n, n_events, zero_head, zero_tail, quantum=None):
    """Smoothed |N(0,1)| noise with Gaussian pulses, zero runs at both ends."""
    x = np.abs(rng.standard_normal(n + 24))
    x = np.convolve(x, np.ones(25) / 25, mode="valid")[:n] * 10.0
    t = np.arange(n)
    for t0 in rng.integers(zero_head + 50, n - zero_tail - 50, size=n_events):
        x += rng.uniform(5, 20) * np.exp(-0.5 * ((t - t0) / 6.0) ** 2)
    if quantum:
        x = np.round(x / quantum) * quantum
    x[:zero_head] = 0.0
    if zero_tail:
        x[-zero_tail:] = 0.0
    return x.astype(np.float32)


def cases(rng):
    out = {}
    out["rms_even"] = (beam_like(rng, 20000, 12, 40, 1500), 3000, 0.66, "rms", 3.0, 300)
    out["rms_odd"] = (beam_like(rng, 15001, 8, 0, 900), 2501, 0.5, "rms", 2.5, 120)
    out["mad_even"] = (beam_like(rng, 20000, 12, 10, 1500), 3000, 0.66, "mad", 8.0, 300)
    out["mad_odd"] = (beam_like(rng, 12345, 6, 0, 700), 1999, 0.66, "mad", 6.0, 77.5)
    # negative values before the zero tail: a rising edge into a zero plateau
    x = beam_like(rng, 9000, 5, 0, 800) - 3.0
    x[-800:] = 0.0
    out["negative_zero_plateau"] = (x, 1000, 0.66, "rms", 4.0, 50)
    # quantised values: many plateaus and equal heights (no minimum distance)
    out["plateaus"] = (beam_like(rng, 6000, 10, 0, 0, quantum=0.5), 1500, 0.66, "mad", 3.0, None)
    out["short_window"] = (beam_like(rng, 700, 3, 0, 20), 64, 0.9, "rms", 1.0, 5)
    # the reference's own beam_max of the 4,000-source network (strict rule)
    bm = np.load(os.path.join(HERE, "tutorial_scale.npz"))["beam_max_strict"]
    out["tutorial_scale_beam"] = (bm.astype(np.float32), 1200, 0.66, "rms", 4.0, 150)
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BEAMPOWER_REFERENCE")
    if not ref_root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> "
                 "(or set BEAMPOWER_REFERENCE)")
    tdt = load_threshold_function(ref_root)
    rng = np.random.default_rng(2024)
    for i, (name, (x, W, ov, kind, nd, dist)) in enumerate(cases(rng).items()):
        n_zeros = int((x == 0.0).sum())
        np.random.seed(1000 + i)
        noise = np.random.normal(size=n_zeros).astype("float32")
        np.random.seed(1000 + i)
        thr = tdt(x, W, overlap=ov, threshold_type=kind, num_dev=nd)
        peaks = signal.find_peaks(x, distance=dist)[0]
        det = peaks[x[peaks] > thr[peaks]]
        np.savez_compressed(os.path.join(HERE, f"detection_{name}.npz"), x=x, noise=noise,
                            window=W, overlap=ov, kind=kind, num_dev=nd,
                            distance=-1.0 if dist is None else float(dist),
                            threshold=thr.astype(np.float32), peaks=peaks, detections=det)
        print(f"wrote {name}: n={x.size} zeros={n_zeros} peaks={peaks.size} det={det.size}")


if __name__ == "__main__":
    main()
