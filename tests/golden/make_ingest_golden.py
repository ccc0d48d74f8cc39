"""Generate tests/golden/ingest.npz from the reference tutorial itself.

Runs the tutorial cell that defines ``sec_to_samp``
(notebooks/3_beampower.ipynb:378-393) from the reference checkout and stores
seeded travel times (seconds) with their sample delays, absolute and
relative to each source's earliest arrival (:396), at two sampling rates.

    python tests/golden/make_ingest_golden.py [reference checkout]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NOTEBOOK = "notebooks/3_beampower.ipynb"


def load_sec_to_samp(ref_root):
    nb = json.load(open(os.path.join(ref_root, NOTEBOOK)))
    for cell in nb["cells"]:
        src = "".join(cell["source"])
        if cell["cell_type"] == "code" and "def sec_to_samp" in src:
            ns = {"np": np}
            exec(compile(src.split("\nsampling_rate =")[0], NOTEBOOK, "exec"), ns)
            return ns["sec_to_samp"]
    raise RuntimeError("sec_to_samp not found in " + NOTEBOOK)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BEAMPOWER_REFERENCE")
    if not ref_root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> "
                 "(or set BEAMPOWER_REFERENCE)")
    f = load_sec_to_samp(ref_root)
    rng = np.random.default_rng(99)
    tt = rng.uniform(0.0, 60.0, size=(300, 12, 2)).astype(np.float32)
    # values whose product with the rate lands near an integer
    tt[0, :, 0] = (np.arange(12) / 25.0).astype(np.float32)
    tt[1, :, 0] = ((np.arange(12) + 0.79) / 25.0).astype(np.float32)
    tt[2, :, :] = -tt[2, :, :]
    tt[3, 0, 0], tt[3, 1, 0], tt[3, 2, 0] = 0.0, -0.0, 1e9
    tt[3, 3, 0], tt[3, 4, 0], tt[3, 5, 0] = np.nan, np.inf, -np.inf
    res = {"seconds": tt}
    with np.errstate(invalid="ignore"):
        for sr in (25.0, 100.0):
            d = f(tt, sr)
            res[f"delays_{int(sr)}"] = d
            rel = d.copy()
            rel -= np.min(rel, axis=(1, 2), keepdims=True)
            res[f"relative_{int(sr)}"] = rel
    np.savez_compressed(os.path.join(HERE, "ingest.npz"), **res)
    print("wrote ingest.npz")


if __name__ == "__main__":
    main()
