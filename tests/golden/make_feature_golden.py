"""Generate tests/golden/features.npz from the reference tutorial itself.

The envelope feature of the tutorial (notebooks/3_beampower.ipynb:74-103,
``envelope``) lives in a notebook cell.  This script reads the notebook from
the reference checkout, runs that cell in a namespace holding the names the
notebook imports for it (numpy, scipy.signal, scipy.stats'
median_abs_deviation), and stores, per seeded trace, the input, the
feature, and the raw envelope ``np.abs(signal.hilbert(x))`` (the scale the
GPU test's tolerance is stated against).

    python tests/golden/make_feature_golden.py [reference checkout]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
from scipy import signal
from scipy.stats import median_abs_deviation

HERE = os.path.dirname(os.path.abspath(__file__))
NOTEBOOK = "notebooks/3_beampower.ipynb"


def load_envelope(ref_root):
    nb = json.load(open(os.path.join(ref_root, NOTEBOOK)))
    for cell in nb["cells"]:
        src = "".join(cell["source"])
        if cell["cell_type"] == "code" and "def envelope" in src:
            ns = {"np": np, "signal": signal, "scimad": median_abs_deviation}
            exec(compile(src, NOTEBOOK, "exec"), ns)
            return ns["envelope"]
    raise RuntimeError("envelope not found in " + NOTEBOOK)


def traces(rng):
    out = {}

    def seismic(n, n_events):
        x = rng.standard_normal(n).astype(np.float32)
        t = np.arange(n)
        for t0 in rng.integers(50, n - 50, size=n_events):
            x += (rng.uniform(5, 40) * np.exp(-0.5 * ((t - t0) / 8.0) ** 2)
                  * np.sin(0.7 * (t - t0))).astype(np.float32)
        return x

    out["even_1000"] = seismic(1000, 3)
    out["odd_1001"] = seismic(1001, 3)
    out["prime_997"] = seismic(997, 2)
    out["tutorial_6000"] = seismic(6000, 6)
    out["pow2_4096"] = seismic(4096, 4)
    x = (1e-3 * rng.standard_normal(3000)).astype(np.float32)
    x[1500] = 2e3  # normalised envelope far above 1e5: clipped
    out["spike_clipped"] = x
    out["zeros"] = np.zeros(512, np.float32)
    out["short_2"] = np.array([1.0, -2.0], np.float32)
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BEAMPOWER_REFERENCE")
    if not ref_root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> "
                 "(or set BEAMPOWER_REFERENCE)")
    envelope = load_envelope(ref_root)
    res = {}
    for name, x in traces(np.random.default_rng(77)).items():
        feat = envelope(x)
        res[f"x_{name}"] = x
        res[f"feature_{name}"] = np.asarray(feat, np.float32)
        res[f"raw_{name}"] = np.abs(signal.hilbert(x)).astype(np.float32)
        print(f"{name}: n={x.size} feature max {float(np.max(feat)):.4g}")
    np.savez_compressed(os.path.join(HERE, "features.npz"), **res)


if __name__ == "__main__":
    main()
