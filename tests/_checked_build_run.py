"""Run by tests/test_gpu_checked_build.py in a child process whose
BEAMPOWER_B200_LIBRARY names the index-checked library: every call below
would raise (the status word read after the kernel) if a bounds or
alignment check of the staged kernel failed; FP32 results must still equal
the reference fixtures bit for bit.  Prints CHECKED OK at the end."""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32).copy()
    a[np.isnan(a)] = np.float32(np.nan)
    return a.view(np.uint32)


def main():
    import torch
    import beampower_b200 as bp
    from beampower_b200.batch import Window, WindowBatch
    from beampower_b200.synthetic import SMALL, make_workload
    from beampower_b200.tables import TravelTimeTable
    lib = bp.load_library("gpu")
    assert lib._name.endswith("libbeampower_b200_checked.so"), lib._name
    n_calls = 0
    for path in sorted(glob.glob(os.path.join(HERE, "golden", "small_*.npz"))):
        g = dict(np.load(path))
        F, A, D, W = g["F"], g["A"], g["D"], g["W"]
        for oob in ("strict", "flexible"):
            if f"beam_max_{oob}" in g:
                bm, am = bp.beamform(F, D, A, W, reduce="max", out_of_bounds=oob)
                assert np.array_equal(bits(bm), bits(g[f"beam_max_{oob}"])), (path, oob)
                assert np.array_equal(am, g[f"argmax_{oob}"]), (path, oob)
                n_calls += 1
            beam = bp.beamform(F, D, A, W, reduce=None, out_of_bounds=oob)
            ok = g[f"beam_{oob}"] != 0
            assert np.array_equal(bits(beam[ok]), bits(g[f"beam_{oob}"][ok])), (path, oob)
            n_calls += 1
            if np.isfinite(W).all():
                for storage in ("fp16", "bf16"):
                    bp.beamform(F, D, A, W, reduce="max", out_of_bounds=oob, storage=storage)
                    n_calls += 1
    # the 4,000-source network, every storage, both rules
    wl = make_workload(SMALL)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    for storage in ("fp32", "fp16", "bf16"):
        for oob in ("strict", "flexible"):
            bp.beamform(F, D, A, W, reduce="max", out_of_bounds=oob, storage=storage)
            n_calls += 1
    # a persistent batch over two windows with a station subset (status word read back)
    table = TravelTimeTable(D, W)
    batch = WindowBatch([table], [Window(0, 6000), Window(0, 3500, stations=range(0, 20, 2))],
                        A, storage="bf16")
    batch.set_features(0, F)
    batch.set_features(1, F[:, :, :3500])
    batch.run()
    torch.cuda.synchronize()
    assert batch.status() == 0, batch.status()
    batch.close()
    table.close()
    print(f"CHECKED OK ({n_calls + 1} calls)")


if __name__ == "__main__":
    main()
