"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own CPU library (beampower/src/beamform.c compiled into
oracle/_ref/beamform_cpu.so by oracle/Makefile, called with the argument
order of beampower/core.py) on seeded inputs and stores inputs and outputs:

* ``small_<case>.npz``  -- small edge cases, inputs and outputs stored;
* ``tutorial_scale.npz`` -- the 4,000-source / 20-station / 6,000-sample
  network of beampower_b200.synthetic.SMALL: outputs plus a digest of the
  regenerated inputs (the inputs are too large to commit).

The reference is read from its checkout only here, when the fixtures are
(re)generated; tests read the committed .npz files.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference, build  # noqa: E402
from beampower_b200.synthetic import SMALL, digest, make_workload  # noqa: E402


def random_case(rng, n_src, n_sta, n_ch, n_ph, n_t, dmax, zero_frac=0.0, negative=False):
    F = np.abs(rng.standard_normal((n_sta, n_ch, n_t))).astype(np.float32)
    A = rng.uniform(0.0, 1.5, size=(n_sta, n_ch, n_ph)).astype(np.float32)
    lo = -dmax // 3 if negative else 0
    D = rng.integers(lo, dmax + 1, size=(n_src, n_sta, n_ph)).astype(np.int32)
    W = rng.uniform(0.25, 2.0, size=(n_src, n_sta)).astype(np.float32)
    if zero_frac:
        W[rng.random(W.shape) < zero_frac] = 0.0
    return F, A, D, W


def cases():
    rng = np.random.default_rng(12345)
    out = {}
    out["random_p2"] = random_case(rng, 200, 7, 3, 2, 600, 150, zero_frac=0.2)
    out["random_p1"] = random_case(rng, 120, 5, 2, 1, 500, 90)
    out["random_p3"] = random_case(rng, 130, 6, 3, 3, 513, 60, zero_frac=0.1)
    out["random_p5"] = random_case(rng, 70, 4, 2, 5, 300, 40)
    # delays near and beyond the record length, many zero weights
    F, A, D, W = random_case(rng, 150, 6, 3, 2, 400, 500, zero_frac=0.4)
    out["long_delays"] = (F, A, D, W)
    # ties: identical sources repeated (lowest index must win)
    F, A, D, W = random_case(rng, 40, 5, 3, 2, 600, 80)
    D[20:] = D[:20]
    W[20:] = W[:20]
    out["ties"] = (F, A, D, W)
    # NaN in a station that every source masks
    F, A, D, W = random_case(rng, 90, 6, 3, 2, 500, 70)
    F[2, :, 100:140] = np.nan
    W[:, 2] = 0.0
    out["nan_masked_station"] = (F, A, D, W)
    # a source whose weights are all zero, and tiny record
    F, A, D, W = random_case(rng, 33, 3, 1, 2, 37, 20)
    W[5] = 0.0
    out["tiny_all_zero_source"] = (F, A, D, W)
    # negative delays: the reference's strict reduce='max' reads outside the
    # trace for them (its `t + min < 0` test is on size_t, beamform.c:281), so
    # that output is not stored; the other paths are well defined.
    out["negative_delays"] = random_case(rng, 120, 5, 3, 2, 450, 90, negative=True)
    return out


def main():
    build()
    ref = Reference()
    for name, (F, A, D, W) in cases().items():
        U = ref.prestack(F, A)
        res = {"F": F, "A": A, "D": D, "W": W, "U": U}
        for oob, tag in ((0, "strict"), (1, "flexible")):
            if not (oob == 0 and D.min() < 0):
                bm, am = ref.beamform_max(U, D, W, oob)
                res[f"beam_max_{tag}"] = bm
                res[f"argmax_{tag}"] = am
            res[f"beam_{tag}"] = ref.beamform(U, D, W, oob)
        res["differential"] = ref.beamform_differential(U, D, W)
        np.savez_compressed(os.path.join(HERE, f"small_{name}.npz"), **res)
        print("wrote", name)
    wl = make_workload(SMALL)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    U = ref.prestack(F, A)
    res = {"digest": np.array(digest(F, A, D, W)), "events": np.array(wl["events"]),
           "U_digest": np.array(digest(U))}
    for oob, tag in ((0, "strict"), (1, "flexible")):
        bm, am = ref.beamform_max(U, D, W, oob)
        res[f"beam_max_{tag}"] = bm
        res[f"argmax_{tag}"] = am
    np.savez_compressed(os.path.join(HERE, "tutorial_scale.npz"), **res)
    print("wrote tutorial_scale")


if __name__ == "__main__":
    main()
