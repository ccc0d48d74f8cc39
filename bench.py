"""Benchmark of the beamforming hot path (one JSON line on rank 0).

Workload: the plain method at scale -- 400,000 sources, 60 stations,
2 phases, 180,000 samples (1 h at 50 Hz), seeded synthetic data
(beampower_b200.synthetic.LARGE), reduce='max', out_of_bounds='strict',
FP32 storage.  Metric: nominal beam terms per second,
sources x samples x stations x phases.

One step = one full call of the hot path on inputs already in HBM: GPU
prestack of the (S, 3, T) features, table build from the (N, S, P) delays and
(N, S) weights, the staged shift-and-stack kernel with fused max/argmax, and
the key decode.  Inputs (418 MB) are larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``--impl reference`` times the reference's own C/OpenMP library (compiled
from its sources into oracle/_ref/) on the host cores, on a bounded
source sample of the same workload.  Multi-GPU runs are replicas: every rank
processes the whole workload (the benchmark is quoted on one GPU and the path
has no exchange between GPUs).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from beampower_b200.replicas import barrier, max_over_ranks  # noqa: E402
from beampower_b200.synthetic import LARGE, make_workload, nominal_terms  # noqa: E402

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "beam_window_kernel_large.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--out-of-bounds", default="strict", choices=["strict", "flexible"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--n-sources", type=int, default=None,
                    help="keep only the first n sources (profiling runs on a smaller case)")
    ap.add_argument("--storage", default=None, choices=["fp32", "bf16", "fp16"],
                    help="trace storage (default: fp32 for the large workload, fp16 for "
                         "batch and serving)")
    ap.add_argument("--workload", default="large",
                    choices=["large", "batch", "serving", "stages", "shapes"],
                    help="large: the 400k-source plain call (default); batch: 128 windows "
                         "in one persistent launch vs one call per window; serving: "
                         "8 streamed networks with Poisson chunk arrivals; stages: the "
                         "tutorial's steps either side; shapes: every kernel shape timed by "
                         "the autotuner on the 400k table and on a 50k batch table")
    ap.add_argument("--windows", type=int, default=128, help="batch workload: windows")
    ap.add_argument("--duration", type=float, default=3.0,
                    help="serving workload: seconds of arrivals")
    ap.add_argument("--sharded", action="store_true",
                    help="split the sources over the ranks (strong scaling, one NCCL max "
                         "all-reduce of the packed keys per call) instead of replicas")
    ap.add_argument("--max-inflight", type=int, default=8,
                    help="serving workload: chunks admitted to the GPU at once")
    ap.add_argument("--rate-scale", type=float, default=1.0,
                    help="serving workload: arrival rate relative to ~200 chunks/s")
    ap.add_argument("--profile", action="store_true",
                    help="timed steps only: no end-to-end pass, no baselines")
    return ap.parse_args()


def large_config(N, S, P, T, out_of_bounds, storage):
    """The `config` of the large workload, the same in both arms."""
    return {"workload": LARGE.name, "n_sources": N, "n_stations": S, "n_phases": P,
            "n_samples": T, "reduce": "max", "out_of_bounds": out_of_bounds,
            "storage": storage, "parallelism": "replicas",
            "l2": "inputs 418 MB > L2, no flush"}


def effective_terms(D, W, T, flexible):
    """Terms the reference actually computes: weighted (station, phase) pairs
    times the samples the validity rule keeps."""
    P = D.shape[2]
    mask = W != 0
    n_w = mask.sum(axis=1).astype(np.int64)
    if flexible:
        # every sample, but only in-range terms: count per (source, station, phase)
        valid = np.clip(T - np.abs(D.astype(np.int64)), 0, T) * mask[:, :, None]
        return int(valid.sum())
    big = np.iinfo(np.int32).max
    dmin = np.where(mask[:, :, None], D, big).min(axis=(1, 2)).astype(np.int64)
    dmax = np.where(mask[:, :, None], D, -big).max(axis=(1, 2)).astype(np.int64)
    nt = np.clip(T - np.maximum(dmax, 0) - np.maximum(-dmin, 0), 0, T)
    nt[n_w == 0] = 0
    return int((nt * n_w * P).sum())


def algorithmic_hbm_bytes(S, C, P, T, N):
    """HBM bytes a call must move at least: features in, traces out and in,
    delays and weights in, keys out."""
    return 4 * S * C * T + 2 * 4 * S * P * T + 4 * N * S * P + 4 * N * S + 8 * T


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU legs (the reference's C library; the only place bench.py runs oracle/)
# ----------------------------------------------------------------------------

def _cpu_sample(wl, n_sub):
    """Every k-th source of the workload, full record length."""
    N = wl["time_delays"].shape[0]
    stride = max(1, N // n_sub)
    idx = np.arange(0, N, stride)[:n_sub]
    return (np.ascontiguousarray(wl["time_delays"][idx]),
            np.ascontiguousarray(wl["weights_sources"][idx]))


def time_reference_cpu(wl, oob, target_s, threads):
    """Reference prestack + beamform_max on a source sample sized for about
    target_s seconds.  Returns (terms/s, seconds, sources in sample)."""
    from oracle.oracle import Reference, Oracle
    kind = "reference"
    try:
        impl = Reference()
    except OSError:
        impl, kind = Oracle(), "port"
    F, A = wl["waveform_features"], wl["weights_phases"]
    S, C, T = F.shape
    P = A.shape[2]

    def run(n_sub):
        D, W = _cpu_sample(wl, n_sub)
        t0 = time.perf_counter()
        U = impl.prestack(F, A, threads)
        impl.beamform_max(U, D, W, oob, threads)
        return time.perf_counter() - t0, D.shape[0]

    n_sub = 64
    dt, n = run(n_sub)
    while dt < 1.0 and n_sub < wl["time_delays"].shape[0]:
        n_sub *= 4
        dt, n = run(n_sub)
    n_sub = int(min(wl["time_delays"].shape[0], max(1, n_sub * target_s / max(dt, 1e-3))))
    if target_s > 2 * dt:
        dt, n = run(n_sub)
    rate = nominal_terms(n, T, S, P) / dt
    return rate, dt, n, kind


def ref_gpu_baseline(wl, target_s=20.0):
    """The reference's own CUDA path (oracle/_ref/beamform_gpu.so, built for
    sm_100a) on one GPU, reduce='max', strict, on a source sample; run in a
    child process (the library resets OpenMP thread counts)."""
    from oracle.oracle import REF_GPU_SO
    if not os.path.exists(REF_GPU_SO):
        return {"unavailable": "oracle/_ref/beamform_gpu.so not built"}
    code = r"""
import sys, time, json, ctypes as ct, numpy as np
sys.path.insert(0, %r)
from oracle.oracle import Reference, REF_GPU_SO
from beampower_b200.synthetic import LARGE, make_workload
wl = make_workload(LARGE)
F, A, D, W = wl["waveform_features"], wl["weights_phases"], wl["time_delays"], wl["weights_sources"]
U = np.ascontiguousarray(Reference().prestack(F, A, -1))
S, T, P = U.shape
# Masked stations (weight 0) are not skipped by the reference's CUDA kernel
# (beamform.cu:109-115): clamp their delays to the source's weighted minimum so
# that every read stays inside the trace array (output-neutral on the CPU path).
mask = W != 0
big = np.iinfo(np.int32).max
dmin = np.where(mask[:, :, None], D, big).min(axis=(1, 2))
dmin = np.where(dmin == big, 0, dmin).astype(np.int32)
D = np.where(mask[:, :, None], D, dmin[:, None, None]).astype(np.int32)
lib = ct.CDLL(REF_GPU_SO)
f32p, i32p, sz = ct.POINTER(ct.c_float), ct.POINTER(ct.c_int), ct.c_size_t
lib.beamform_max.argtypes = [f32p, i32p, f32p, sz, sz, sz, sz, ct.c_int, f32p, i32p]
lib.beamform_max.restype = None
def run(n):
    stride = max(1, D.shape[0] // n)
    idx = np.arange(0, D.shape[0], stride)[:n]
    d = np.ascontiguousarray(D[idx]); w = np.ascontiguousarray(W[idx])
    bm = np.zeros(T, np.float32); am = np.zeros(T, np.int32)
    t0 = time.perf_counter()
    lib.beamform_max(U.ctypes.data_as(f32p), d.ctypes.data_as(i32p), w.ctypes.data_as(f32p),
                     T, len(idx), S, P, 0, bm.ctypes.data_as(f32p), am.ctypes.data_as(i32p))
    return time.perf_counter() - t0, len(idx)
run(256)
n = 1024
dt, m = run(n)
n = int(min(D.shape[0], max(256, n * %f / max(dt, 1e-3))))
dt, m = run(n)
print(json.dumps({"value": m * T * S * P / dt, "seconds": dt, "sources": m}))
""" % (ROOT, target_s)
    try:
        out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                             timeout=600)
        line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
        if out.returncode != 0 or not line:
            return {"unavailable": f"exit {out.returncode}: {out.stderr.strip()[-200:]}"}
        r = json.loads(line[-1])
        return {"value": r["value"], "unit": "beam terms/s",
                "sample": f"{r['sources']} of 400000 sources (every k-th), all 180000 samples, "
                          f"strict, {r['seconds']:.1f} s, end-to-end incl. H2D",
                "kind": "reference CUDA (beamform.cu, sm_100a build, 1 GPU)"}
    except subprocess.TimeoutExpired:
        return {"unavailable": "timed out"}


_SAMPLED_CHILD = r"""
import sys, json, time, ctypes as ct
import numpy as np
sys.path.insert(0, %r)
from oracle.oracle import Reference, REF_GPU_SO
job = json.loads(sys.argv[1])
ref = Reference()
if job["kind"] == "batch":
    from beampower_b200.synthetic import make_batch_workload, window_features
    wl = make_batch_workload()
    A = wl["weights_phases"]

    def item(i):
        w = wl["windows"][i]
        D, W = wl["grids"][w["table"]]
        m = np.zeros(W.shape[1], np.float32)
        m[w["stations"]] = 1.0
        return window_features(wl, i), A, D, W * m[None, :], len(w["stations"]), w["n_samples"]
else:
    from beampower_b200.synthetic import make_serving_networks, serving_record
    nets = make_serving_networks()

    def item(i):
        n = nets[i]
        D, W = n["delays"], n["weights"]
        lag = int(D.max())
        F, _ = serving_record(n, 2)
        L = n["chunk"]
        # one chunk's record: the chunk plus the max-delay halo it needs
        return (np.ascontiguousarray(F[:, :, :L + lag]), n["weights_phases"], D, W,
                n["n_stations"], L)
gpu = job["mode"] == "gpu"
if gpu:
    lib = ct.CDLL(REF_GPU_SO)
    f32p, i32p, sz = ct.POINTER(ct.c_float), ct.POINTER(ct.c_int), ct.c_size_t
    lib.beamform_max.argtypes = [f32p, i32p, f32p, sz, sz, sz, sz, ct.c_int, f32p, i32p]
    lib.beamform_max.restype = None


def run(F, A, D, W, n_sub):
    stride = max(1, D.shape[0] // n_sub)
    idx = np.arange(0, D.shape[0], stride)[:n_sub]
    d = np.ascontiguousarray(D[idx])
    w = np.ascontiguousarray(W[idx])
    if not gpu:
        t0 = time.perf_counter()
        U = ref.prestack(F, A, -1)
        ref.beamform_max(U, d, w, 0, -1)
        return time.perf_counter() - t0, len(idx)
    U = np.ascontiguousarray(ref.prestack(F, A, -1))
    S, T, P = U.shape
    # masked stations are read by the reference CUDA kernel (beamform.cu:109-115):
    # clamp their delays into the trace (output-neutral for the CPU semantics)
    mask = w != 0
    big = np.iinfo(np.int32).max
    dmin = np.where(mask[:, :, None], d, big).min(axis=(1, 2))
    dmin = np.where(dmin == big, 0, dmin).astype(np.int32)
    d = np.ascontiguousarray(np.where(mask[:, :, None], d, dmin[:, None, None]).astype(np.int32))
    bm = np.zeros(T, np.float32)
    am = np.zeros(T, np.int32)
    t0 = time.perf_counter()
    lib.beamform_max(U.ctypes.data_as(f32p), d.ctypes.data_as(i32p), w.ctypes.data_as(f32p),
                     T, len(idx), S, P, 0, bm.ctypes.data_as(f32p), am.ctypes.data_as(i32p))
    return time.perf_counter() - t0, len(idx)


items = job["items"]
per_item = job["target_s"] / max(1, len(items))
terms = secs = 0.0
done = []
for i in items:
    F, A, D, W, s_used, t_out = item(i)
    P = D.shape[2]
    dt, m = run(F, A, D, W, 128)
    n_sub = int(min(D.shape[0], max(128, 128 * per_item / max(dt, 1e-4))))
    dt, m = run(F, A, D, W, n_sub)
    terms += float(m) * t_out * s_used * P
    secs += dt
    done.append([int(i), int(m), int(D.shape[0])])
print(json.dumps({"terms": terms, "seconds": secs, "items": done}))
"""


def sampled_reference(kind, mode, items, target_s, timeout=900):
    """The reference's own CPU library (mode 'cpu', all host threads) or its
    CUDA path (mode 'gpu', oracle/_ref/beamform_gpu.so on one GPU, host
    buffers, H2D included) on a sample of batch windows or serving chunks,
    in a child process: each item with an evenly strided source subsample
    sized for about target_s / len(items) seconds.  Returns the nominal beam
    terms per second of the sample (window or chunk terms, the sources the
    sample kept)."""
    from oracle.oracle import REF_CPU_SO, REF_GPU_SO
    so = REF_GPU_SO if mode == "gpu" else REF_CPU_SO
    if not os.path.exists(so):
        return {"unavailable": f"{os.path.relpath(so, ROOT)} not built"}
    job = json.dumps({"kind": kind, "mode": mode, "items": list(items), "target_s": target_s})
    try:
        out = subprocess.run([sys.executable, "-c", _SAMPLED_CHILD % ROOT, job],
                             capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"unavailable": "timed out"}
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    if out.returncode != 0 or not line:
        return {"unavailable": f"exit {out.returncode}: {out.stderr.strip()[-200:]}"}
    r = json.loads(line[-1])
    return {"value": r["terms"] / r["seconds"], "unit": "beam terms/s",
            "sample_terms": r["terms"], "sample_seconds": r["seconds"],
            "items": r["items"]}


# ----------------------------------------------------------------------------

def run_reference_arm(args, rank, world):
    """--impl reference: rank 0 times the reference CPU library."""
    if rank != 0:
        return
    wl = make_workload(LARGE)
    S, C, T = wl["waveform_features"].shape
    N, _, P = wl["time_delays"].shape
    threads = os.cpu_count() or 1
    oob = 0 if args.out_of_bounds == "strict" else 1
    # size one step for ~6 s of CPU work
    rate, dt, n_sub, kind = time_reference_cpu(wl, oob, 6.0, threads)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        from oracle.oracle import Reference, Oracle
        impl = Reference() if kind == "reference" else Oracle()
        D, W = _cpu_sample(wl, n_sub)
        U = impl.prestack(wl["waveform_features"], wl["weights_phases"], threads)
        impl.beamform_max(U, D, W, oob, threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    terms = nominal_terms(n_sub, T, S, P)
    value = terms / statistics.mean(times)
    ms_full = nominal_terms(N, T, S, P) / value * 1e3
    line = {
        "impl": "reference", "metric": "beam terms/s (src x t x sta x phase)",
        "value": value, "unit": "beam terms/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3,
        "ms_per_step_full_workload": ms_full, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": large_config(N, S, P, T, args.out_of_bounds, "fp32"),
        "cpu_baseline": {"value": value, "unit": "beam terms/s", "cores": threads, "kind": kind,
                         "sample": f"{n_sub} of {N} sources (every k-th), all {T} samples, "
                                   "prestack + beamform_max per step (ms_per_step: one "
                                   "sampled step; ms_per_step_full_workload: the whole "
                                   "workload at the same rate)"},
        "e2e": {"value": value, "unit": "beam terms/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import beampower_b200 as bp
    from beampower_b200.core import check, load_library
    from beampower_b200.tables import TravelTimeTable, _stream_ptr

    dist = world > 1
    if dist:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = load_library("gpu")
    oob = 0 if args.out_of_bounds == "strict" else 1

    wl = make_workload(LARGE)
    if args.n_sources:
        wl["time_delays"] = np.ascontiguousarray(wl["time_delays"][:args.n_sources])
        wl["weights_sources"] = np.ascontiguousarray(wl["weights_sources"][:args.n_sources])
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    S, C, T = F.shape
    N, _, P = D.shape
    terms = nominal_terms(N, T, S, P)
    eff = effective_terms(D, W, T, oob == 1)

    dF = torch.from_numpy(F).to(dev)
    dA = torch.from_numpy(A).to(dev)
    dD = torch.from_numpy(D).to(dev)
    dW = torch.from_numpy(W).to(dev)
    stream = torch.cuda.current_stream()

    # peaks of this GPU at its current clock (binding roofline of the kernel)
    smem_gbs, fp32_tf = ctypes_double(), ctypes_double()
    check(lib.bp_measure_peaks(_stream_ptr(), smem_gbs.ref, fp32_tf.ref))

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step(record):
        # one full call; its traces and outputs are dropped at the end of the
        # step (stream-ordered), as a caller's loop drops them, so that the
        # next step reuses torch's cached blocks instead of allocating anew
        e0, e1, e2, e3 = ev(), ev(), ev(), ev()
        e0.record(stream)
        table = TravelTimeTable(dD, dW, device=dev)
        e1.record(stream)
        traces = table.traces_from_features(dF, dA, storage=args.storage)
        e2.record(stream)
        bm, am = table.beamform_max(traces, oob)
        e3.record(stream)
        record.append((e0, e1, e2, e3, table))
        del traces, bm, am

    # warm-up
    recs = []
    for _ in range(args.warmup):
        step(recs)
    torch.cuda.synchronize()
    for r in recs:
        r[4].close()
    recs = []
    launches0 = lib.bp_launch_count()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    barrier(dev)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.5)
    t_start, t_end = ev(), ev()
    t_start.record(stream)
    for _ in range(args.steps):
        step(recs)
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    launches = lib.bp_launch_count() - launches0
    elapsed_ms = t_start.elapsed_time(t_end)
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    table_ms = statistics.mean(r[0].elapsed_time(r[1]) for r in recs)
    prestack_ms = statistics.mean(r[1].elapsed_time(r[2]) for r in recs)
    kernel_ms = statistics.mean(r[2].elapsed_time(r[3]) for r in recs)
    info = recs[0][4].info
    # the other trace storage types on the same resident table (kernel only)
    variants = {}
    run_variants = {}
    if not args.profile:
        vt = recs[-1][4]
        for stg in ("fp32", "fp16", "bf16"):
            if stg == args.storage:
                continue
            tr = vt.traces_from_features(dF, dA, storage=stg)
            vt.beamform_max(tr, oob)
            e0, e1 = ev(), ev()
            e0.record(stream)
            for _ in range(2):
                vt.beamform_max(tr, oob)
            e1.record(stream)
            torch.cuda.synchronize()
            kms = e0.elapsed_time(e1) / 2
            variants[stg] = {"kernel_ms": kms, "value": terms / (kms * 1e-3),
                             "unit": "beam terms/s", "kernel_config":
                             lib.bp_get_kernel_config({"fp32": 0, "bf16": 1, "fp16": 2}[stg], 1)}
            del tr
        # the other runs of the same configuration: the flexible rule, and
        # reduce='none' on the first 20,000 sources (a 20,000 x T beam)
        tr = vt.traces_from_features(dF, dA, storage="fp32")
        flex = 1 - oob
        vt.beamform_max(tr, flex)
        e0, e1 = ev(), ev()
        e0.record(stream)
        vt.beamform_max(tr, flex)
        e1.record(stream)
        torch.cuda.synchronize()
        kms = e0.elapsed_time(e1)
        eff_f = effective_terms(D, W, T, flex == 1)
        run_variants["flexible" if flex else "strict"] = {
            "kernel_ms": kms, "value": terms / (kms * 1e-3), "unit": "beam terms/s",
            "effective_terms": eff_f, "smem_frac": (eff_f * 4 / (kms * 1e-3)) / (smem_gbs.value * 1e9),
            "storage": "fp32"}
        del tr
        n_sub = min(20000, N)
        sub = TravelTimeTable(dD[:n_sub].contiguous(), dW[:n_sub].contiguous(), device=dev)
        tr = sub.traces_from_features(dF, dA, storage="fp32")
        beam = torch.zeros((n_sub, T), dtype=torch.float32, device=dev)
        sub.beamform(tr, oob, out=beam)
        e0, e1 = ev(), ev()
        e0.record(stream)
        sub.beamform(tr, oob, out=beam)
        e1.record(stream)
        torch.cuda.synchronize()
        kms = e0.elapsed_time(e1)
        sub_terms = nominal_terms(n_sub, T, S, P)
        out_bytes = n_sub * T * 4
        run_variants["reduce_none_20k"] = {
            "kernel_ms": kms, "value": sub_terms / (kms * 1e-3), "unit": "beam terms/s",
            "n_sources": n_sub, "output_bytes": out_bytes,
            "output_gbs": out_bytes / (kms * 1e-3) / 1e9, "storage": "fp32"}
        del beam, tr
        sub.close()
    for r in recs:
        r[4].close()
    ms_per_step = elapsed_ms / args.steps
    value = world * terms / (ms_per_step * 1e-3)

    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms_per_step,
                              "kernel_ms": kernel_ms, "table_ms": table_ms,
                              "prestack_ms": prestack_ms, "n_sources": N,
                              "storage": args.storage, "table": info}), flush=True)
        if dist:
            tdist.destroy_process_group()
        return

    # ---- end to end through the public numpy API: host inputs copied in and
    # results copied out inside the timed region, on pageable arrays (what
    # the reference's callers pass, beampower.py:108-110) and on pinned ones
    def e2e(hF, hD, hA, hW):
        bp.beamform(hF, hD, hA, hW, reduce="max", out_of_bounds=args.out_of_bounds,
                    storage=args.storage)
        times = []
        for _ in range(max(2, min(args.steps, 3))):
            barrier(dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bp.beamform(hF, hD, hA, hW, reduce="max", out_of_bounds=args.out_of_bounds,
                        storage=args.storage)
            times.append(time.perf_counter() - t0)
        return max_over_ranks(statistics.mean(times), dev)

    e2e_s = e2e(F, D, A, W)
    pin = {k: torch.from_numpy(v).pin_memory() for k, v in
           (("F", F), ("A", A), ("D", D), ("W", W))}
    e2e_pinned_s = e2e(*(pin[k].numpy() for k in ("F", "D", "A", "W")))
    h2d = F.nbytes + A.nbytes + D.nbytes + W.nbytes
    d2h = 8 * T

    line = None
    if rank == 0:
        # roofline of the dominant kernel: shared-memory operand delivery,
        # 4 B of trace per effective term
        smem_achieved = eff * 4 / (kernel_ms * 1e-3) / 1e9
        traffic = None
        if os.path.exists(PROFILE_TRAFFIC):
            with open(PROFILE_TRAFFIC) as fh:
                prof = json.load(fh)
            traffic = prof.get("dram_bytes_per_launch_full_size")
        hbm_peak = None
        if os.path.exists(MEASURED_PEAKS):
            with open(MEASURED_PEAKS) as fh:
                hbm_peak = json.load(fh).get("hbm_gbs")
        hbm_bytes = algorithmic_hbm_bytes(S, C, P, T, N)
        line = {
            "metric": "beam terms/s (src x t x sta x phase)",
            "value": value,
            "unit": "beam terms/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": large_config(N, S, P, T, args.out_of_bounds, args.storage),
            "effective_terms_per_step": eff,
            "nominal_terms_per_step": terms,
            "breakdown_ms": {"table_build": table_ms, "prestack": prestack_ms,
                             "beam_kernel_and_decode": kernel_ms},
            "roofline": {
                "bound": "smem",
                "achieved": smem_achieved,
                "peak": smem_gbs.value,
                "unit": "GB/s",
                "frac": smem_achieved / smem_gbs.value,
                "traffic": traffic,
                "note": "shared-memory operand roof (4 B of trace per effective term), peak "
                        "measured live by bp_measure_peaks; FP32 and HBM views below",
                "fp32_view": {"achieved_tflops": eff * 2 / (kernel_ms * 1e-3) / 1e12,
                              "peak_tflops": fp32_tf.value},
                "hbm_view": {"achieved_gbs": hbm_bytes / (ms_per_step * 1e-3) / 1e9,
                             "peak_gbs": hbm_peak, "of": "measured (MEASURED_PEAKS.json)"},
            },
            "table": info,
            "storage_variants": variants,
            "run_variants": run_variants,
            "e2e": {"value": world * terms / e2e_s, "unit": "beam terms/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "seconds_per_step": e2e_s, "host_inputs": "pageable numpy arrays",
                    "pinned": {"value": world * terms / e2e_pinned_s,
                               "seconds_per_step": e2e_pinned_s}},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
    if dist:
        barrier(dev)
        tdist.destroy_process_group()
    if rank != 0:
        return
    # host-side baselines (rank 0, N = 1 only)
    if world == 1 and not args.no_cpu_baseline:
        rate, dt, n_sub, kind = time_reference_cpu(wl, oob, args.cpu_seconds, os.cpu_count() or 1)
        line["cpu_baseline"] = {
            "value": rate, "unit": "beam terms/s", "cores": os.cpu_count() or 1, "kind": kind,
            "sample": f"{n_sub} of {N} sources (every k-th), all {T} samples, prestack + "
                      f"beamform_max, {dt:.1f} s"}
    if world == 1 and not args.no_ref_gpu:
        line["ref_gpu_baseline"] = ref_gpu_baseline(wl)
    print(json.dumps(line), flush=True)


class ctypes_double:
    def __init__(self):
        import ctypes
        self._v = ctypes.c_double(0.0)
        self.ref = ctypes.byref(self._v)

    @property
    def value(self):
        return self._v.value


def main():
    args = parse()
    if args.storage is None:
        args.storage = "fp16" if args.workload in ("batch", "serving") else "fp32"
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.workload == "batch":
        run_batch(args, local_rank)
        return
    if args.workload == "serving":
        # A serving process loads every kernel when CUDA starts, so that no
        # request pays a module load (with lazy loading, torch's default, a
        # kernel used for the first time inside a request stalled it for
        # tens of ms).  The variable is read when the process starts CUDA:
        # restart with it set.
        if os.environ.get("CUDA_MODULE_LOADING") != "EAGER":
            os.environ["CUDA_MODULE_LOADING"] = "EAGER"
            os.execv(sys.executable, [sys.executable] + sys.argv)
        run_serving(args, local_rank)
        return
    if args.workload == "stages":
        run_stages(args, local_rank)
        return
    if args.workload == "shapes":
        run_shapes(args, local_rank)
        return
    if args.sharded:
        run_sharded(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)



# ----------------------------------------------------------------------------
# Batching and serving workloads (single GPU)
# ----------------------------------------------------------------------------

def run_batch(args, local_rank):
    """128 detection windows (3,000-90,000 samples, 20-80 of 100 stations, a
    400,000- or 50,000-source grid each): one persistent launch replayed from
    a CUDA graph, against (1) this library's plain path called once per
    window (FP32, device inputs), (2) the reference's CUDA path called once
    per window and (3) the reference's C library on the host cores -- (2)
    and (3) on a sample of windows, extrapolated to the whole batch."""
    import torch
    import beampower_b200 as bp
    from beampower_b200.batch import Window, WindowBatch
    from beampower_b200.synthetic import make_batch_workload, window_features_torch
    from beampower_b200.tables import TravelTimeTable
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = make_batch_workload(n_windows=args.windows)
    tables = [TravelTimeTable(D, W, device=dev) for D, W in wl["grids"]]
    windows = [Window(w["table"], w["n_samples"], w["stations"]) for w in wl["windows"]]
    batch = WindowBatch(tables, windows, wl["weights_phases"], storage=args.storage)
    for i in range(len(windows)):
        batch.set_features(i, window_features_torch(wl, i, dev))
    terms = batch.terms()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    batch.capture()
    for _ in range(args.warmup):
        batch.run()
    sampler = ClockSampler(local_rank)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    launches0 = bp.core.launch_count()
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(args.steps):
        batch.run()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms_batch = e0.elapsed_time(e1) / args.steps
    # the plain path, one call per window (device-resident inputs, subset as
    # zero weights, table built per call as a call does)
    A = torch.from_numpy(wl["weights_phases"]).to(dev)
    Dd = [torch.from_numpy(D).to(dev) for D, _ in wl["grids"]]
    plain_ms = []
    for _ in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i, w in enumerate(wl["windows"]):
            W = torch.zeros((Dd[w["table"]].shape[0], wl["spec"].n_stations), device=dev)
            W[:, w["stations"]] = 1.0
            bp.beamform(batch.features[i], Dd[w["table"]], A, W, reduce="max",
                        out_of_bounds="strict", storage="fp32")
        torch.cuda.synchronize()
        plain_ms.append((time.perf_counter() - t0) * 1e3)
    plain = statistics.mean(plain_ms)
    value = terms / (ms_batch * 1e-3)
    # the same batch with the other trace storages (CUDA graph replay, 2 steps)
    variants = {}
    for stg in ("fp32", "fp16", "bf16"):
        if stg == args.storage:
            continue
        vb = WindowBatch(tables, windows, wl["weights_phases"], storage=stg)
        for i in range(len(windows)):
            vb.set_features(i, batch.features[i])
        vb.capture()
        vb.run()
        torch.cuda.synchronize()
        v0, v1 = ev(), ev()
        v0.record()
        for _ in range(2):
            vb.run()
        v1.record()
        torch.cuda.synchronize()
        vms = v0.elapsed_time(v1) / 2
        variants[stg] = {"ms_per_step": vms, "value": terms / (vms * 1e-3),
                         "vs_plain_per_window": plain / vms}
        vb.close()
    line = {
        "metric": "beam terms/s (src x t x sta x phase)", "value": value,
        "unit": "beam terms/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_batch, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.storage == "fp32" else args.storage,
        "data": "synthetic",
        "config": {"workload": wl["spec"].name, "windows": len(windows),
                   "storage": args.storage, "graph": True, "persistent_launch": True,
                   "kernel_config": bp.core.load_library("gpu").bp_get_kernel_config(
                       {"fp32": 0, "bf16": 1, "fp16": 2}[args.storage], 1),
                   "l2": "inputs of every step > L2 (features of 128 windows), no flush"},
        "terms_per_step": terms,
        "storage_variants": variants,
        "gpu_launches": int((bp.core.launch_count() - launches0) / max(1, args.steps)),
        "plain_per_window": {"value": terms / (plain * 1e-3), "ms_per_step": plain,
                             "storage": "fp32",
                             "note": "beampower_b200.beamform per window, device inputs"},
        "clocks": clocks,
    }
    speed = {"vs_plain_per_window": plain / ms_batch}
    sample = list(range(0, len(windows), max(1, len(windows) // 8)))[:8]
    if not args.no_cpu_baseline:
        cpu = sampled_reference("batch", "cpu", sample, args.cpu_seconds)
        if "value" in cpu:
            cpu.update({"cores": os.cpu_count() or 1, "kind": "reference",
                        "ms_per_step_extrapolated": terms / cpu["value"] * 1e3,
                        "sample": f"windows {sample}, strided source subsample each, "
                                  "reference prestack + beamform_max, extrapolated"})
            speed["vs_reference_cpu"] = value / cpu["value"]
        line["cpu_baseline"] = cpu
    if not args.no_ref_gpu:
        rg = sampled_reference("batch", "gpu", sample, 20.0)
        if "value" in rg:
            rg.update({"kind": "reference CUDA (beamform.cu, sm_100a build, 1 GPU) per window",
                       "ms_per_step_extrapolated": terms / rg["value"] * 1e3,
                       "sample": f"windows {sample}, strided source subsample each, "
                                 "end-to-end incl. H2D, extrapolated"})
            speed["vs_reference_gpu_per_window"] = value / rg["value"]
        line["ref_gpu_per_window"] = rg
    line["speedup"] = speed
    print(json.dumps(line), flush=True)
    batch.close()


def run_serving(args, local_rank):
    """8 networks streaming 60 s chunks with Poisson arrivals, resident
    tables, carried halo, continuous batching under a 150 GB budget,
    earliest-deadline-first admission and priority streams.  Capacity is
    estimated from each network's chunk device time alone; p50/p99 latency is
    swept over offered loads of 5-75 % of it (overall and for the
    400,000-source networks alone); the headline throughput is measured at
    the specified ~200 chunks/s (beyond one GPU's capacity)."""
    import gc
    import torch
    from beampower_b200.stream import NetworkStream, StreamScheduler
    from beampower_b200.synthetic import SERVING, make_serving_networks, serving_record
    from beampower_b200.tables import TravelTimeTable
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nets = make_serving_networks()
    pool = 4  # distinct chunks per network, cycled
    streams, chunks = {}, {}
    for n in nets:
        tab = TravelTimeTable(n["delays"], n["weights"], device=dev)
        streams[n["name"]] = NetworkStream(tab, n["weights_phases"], "strict",
                                           storage=args.storage, name=n["name"])
        F, _ = serving_record(n, pool)
        L = n["chunk"]
        chunks[n["name"]] = [torch.from_numpy(F[:, :, i * L:(i + 1) * L].copy()).pin_memory()
                             for i in range(pool)]
    large = {n["name"] for n in nets if n["delays"].shape[0] >= 400000}
    lib = streams[nets[0]["name"]].lib
    st_id = {"fp32": 0, "bf16": 1, "fp16": 2}[args.storage]
    net_info = {n["name"]: {"n_sources": int(n["delays"].shape[0]),
                            "n_stations": n["n_stations"], "fs": n["fs"], "chunk": n["chunk"],
                            "max_spread": streams[n["name"]].table.info["max_spread"],
                            "max_delay": streams[n["name"]].table.info["max_delay"],
                            "kernel_config": lib.bp_table_kernel_config(
                                streams[n["name"]].table.handle, st_id, 1),
                            "rate": n["rate"]} for n in nets}
    counters = {n["name"]: 0 for n in nets}

    def next_chunk(name):
        c = chunks[name][counters[name] % pool]
        counters[name] += 1
        return c

    # device time of one chunk per network alone (after a warm-up chunk)
    alone_ms = {}
    for n in nets:
        ns = streams[n["name"]]
        ns.push(next_chunk(n["name"]))
        ns.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ns.stream)
        for _ in range(3):
            ns.push(next_chunk(n["name"]))
        e1.record(ns.stream)
        ns.synchronize()
        alone_ms[n["name"]] = e0.elapsed_time(e1) / 3
    busy_per_s = sum(n["rate"] * alone_ms[n["name"]] * 1e-3 for n in nets)  # at rate_scale 1
    cap_scale = 1.0 / busy_per_s  # rate_scale that fills one GPU

    def run_load(scale, duration, max_inflight, seed):
        for ns in streams.values():
            ns.results = []
        rng = np.random.default_rng(seed)
        arrivals = []
        for n in nets:
            t = 0.0
            while True:
                t += rng.exponential(1.0 / (n["rate"] * scale))
                if t > duration:
                    break
                arrivals.append((t, n["name"]))
        arrivals.sort()
        sched = StreamScheduler(streams, max_inflight=max_inflight, memory_budget=150e9,
                                latency_budget=0.05)
        gc.collect()
        gc.disable()  # no collector pauses inside the request loop
        t_start = time.perf_counter()
        k = 0
        while k < len(arrivals) or sched.pending or sched.inflight:
            now = time.perf_counter() - t_start
            while k < len(arrivals) and arrivals[k][0] <= now:
                name = arrivals[k][1]
                sched.submit(name, next_chunk(name), arrival=t_start + arrivals[k][0])
                k += 1
            sched.step()
            time.sleep(5e-5)
        gc.enable()
        st = sched.stats()
        lat_l = np.array([c - a for nm, a, c, *_ in sched.done if nm in large])
        st["large_p50_ms"] = float(np.percentile(lat_l, 50) * 1e3) if lat_l.size else None
        st["large_p99_ms"] = float(np.percentile(lat_l, 99) * 1e3) if lat_l.size else None
        st["large_chunks"] = int(lat_l.size)
        st["offered_chunks_per_s"] = sum(n["rate"] * scale for n in nets)
        return st

    # every network's chunk once through every priority stream (cached memory
    # per stream), then a short run at half the capacity, both untimed
    StreamScheduler(streams).warm_up({n["name"]: next_chunk(n["name"]) for n in nets})
    run_load(0.5 * cap_scale, 1.0, args.max_inflight, seed=7)
    sampler = ClockSampler(local_rank)
    sampler.start()
    curve = []
    for frac in (0.05, 0.10, 0.25, 0.50, 0.75):
        scale = frac * cap_scale
        duration = max(args.duration, 150.0 / (SERVING.total_rate * scale))
        st = run_load(scale, duration, args.max_inflight, seed=int(frac * 1000))
        curve.append({"load_of_capacity": frac, "offered_chunks_per_s": st["offered_chunks_per_s"],
                      "chunks": st["chunks"], "duration_s": duration,
                      "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                      "large_p50_ms": st["large_p50_ms"], "large_p99_ms": st["large_p99_ms"],
                      "large_chunks": st["large_chunks"], "terms_per_s": st["terms_per_s"],
                      "wait_p99_ms": st["wait_p99_ms"], "device_p50_ms": st["device_p50_ms"],
                      "device_p99_ms": st["device_p99_ms"],
                      "enqueue_p50_ms": st["enqueue_p50_ms"],
                      "enqueue_p99_ms": st["enqueue_p99_ms"]})
    st = run_load(args.rate_scale, args.duration, args.max_inflight, seed=1)
    clocks = sampler.stop()
    ok = [c["load_of_capacity"] for c in curve
          if c["large_p99_ms"] is not None and c["large_p99_ms"] < 50.0]
    offered_terms = sum(n["rate"] * args.rate_scale * n["delays"].shape[0] * n["chunk"]
                        * n["n_stations"] * 2 for n in nets)
    value = st.get("terms_per_s")
    line = {
        "metric": "beam terms/s (src x t x sta x phase)", "value": value,
        "unit": "beam terms/s", "n_gpus": 1, "steps": st.get("chunks"), "warmup": 4 * len(nets),
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.storage == "fp32" else args.storage,
        "data": "synthetic",
        "config": {"workload": SERVING.name, "networks": len(nets),
                   "offered_chunks_per_s": st["offered_chunks_per_s"],
                   "offered_terms_per_s": offered_terms, "duration_s": args.duration,
                   "max_inflight": args.max_inflight, "storage": args.storage,
                   "admission": "earliest deadline first (arrival + 50 ms)",
                   "module_loading": os.environ.get("CUDA_MODULE_LOADING"),
                   "streams": "priority pool, oldest chunk in flight highest"},
        "latency_ms": {"p50": st.get("p50_ms"), "p99": st.get("p99_ms"),
                       "max": st.get("max_ms"), "large_p50": st.get("large_p50_ms"),
                       "large_p99": st.get("large_p99_ms")},
        "latency_breakdown_ms": {k: st.get(k) for k in (
            "wait_p50_ms", "wait_p99_ms", "admit_to_start_p50_ms", "admit_to_start_p99_ms",
            "device_p50_ms", "device_p99_ms", "enqueue_p50_ms", "enqueue_p99_ms")},
        "networks": net_info,
        "capacity": {"chunk_device_ms_alone": alone_ms,
                     "chunks_per_s": SERVING.total_rate * cap_scale,
                     "of_specified_load": cap_scale,
                     "large_networks": sorted(large)},
        "load_curve": curve,
        "highest_load_with_large_p99_below_50ms": max(ok) if ok else None,
        "queue": {k: st.get(k) for k in ("peak_queue_depth", "peak_inflight",
                                          "peak_device_bytes_admitted")},
        "per_network": st.get("per_network"),
        "chunks_done": st.get("chunks"), "span_s": st.get("span_s"),
        "clocks": clocks,
    }
    sample = list(range(len(nets)))
    speed = {}
    if not args.no_cpu_baseline:
        cpu = sampled_reference("serving", "cpu", sample, args.cpu_seconds)
        if "value" in cpu:
            cpu.update({"cores": os.cpu_count() or 1, "kind": "reference",
                        "sample": "one 60 s chunk (+ its max-delay halo) of every network, "
                                  "strided source subsample, reference prestack + "
                                  "beamform_max"})
            speed["vs_reference_cpu"] = value / cpu["value"]
        line["cpu_baseline"] = cpu
    if not args.no_ref_gpu:
        rg = sampled_reference("serving", "gpu", sample, 20.0)
        if "value" in rg:
            rg.update({"kind": "reference CUDA (beamform.cu, sm_100a build, 1 GPU) per chunk",
                       "sample": "one 60 s chunk (+ halo) of every network, strided source "
                                 "subsample, end-to-end incl. H2D"})
            speed["vs_reference_gpu_per_chunk"] = value / rg["value"]
        line["ref_gpu_per_chunk"] = rg
    line["speedup"] = speed
    print(json.dumps(line), flush=True)


def run_shapes(args, local_rank):
    """Kernel time of every compiled shape of the staged kernel, per trace
    storage, through the autotuner (beampower_b200.autotune): on the
    400,000-source table of the large workload (60 stations, 180,000
    samples), on the 50,000-source grid of the batch workload (100
    stations) with one 90,000-sample window over all stations, and on a
    regional network whose delay windows are wider than the 16-bit default
    shape holds (64,000 sources, 800 km, 100 Hz, 120,000 samples).  Shapes
    whose shared memory does not fit a table are reported as None."""
    import torch
    from beampower_b200 import autotune
    from beampower_b200.core import load_library
    from beampower_b200.synthetic import (REGIONAL, make_batch_workload, window_features,
                                          nominal_terms)
    from beampower_b200.tables import TravelTimeTable
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = load_library("gpu")
    wl = make_workload(LARGE)
    bw = make_batch_workload(n_windows=1)
    D50, W50 = bw["grids"][1]
    F50 = window_features({**bw, "windows": [{**bw["windows"][0], "table": 1,
                                               "n_samples": 90000, "events": []}]}, 0)
    cases = [("large-400k-src-60-sta-180000-samples", wl["time_delays"], wl["weights_sources"],
              wl["waveform_features"], wl["weights_phases"]),
             ("batch-grid-50k-src-100-sta-90000-samples", D50, W50, F50, bw["weights_phases"])]
    rg = make_workload(REGIONAL)
    cases.append((REGIONAL.name, rg["time_delays"], rg["weights_sources"],
                  rg["waveform_features"], rg["weights_phases"]))
    out = {"shapes": dict(autotune.configs()), "tables": {}}
    sampler = ClockSampler(local_rank)
    sampler.start()
    for name, D, W, F, A in cases:
        table = TravelTimeTable(D, W, device=dev)
        N, S, P = D.shape
        terms = nominal_terms(N, F.shape[2], S, P)
        res = {"terms": terms, "max_spread": table.info["max_spread"],
               "max_active": table.info["max_active"], "storages": {}}
        for stg in ("fp32", "fp16", "bf16"):
            tr = table.traces_from_features(F, A, storage=stg)
            r = autotune.autotune(table, tr, repeats=2, write_cache=False)
            res["storages"][stg] = {"ms": r["times_ms"], "best": r["best"]}
            lib.bp_set_kernel_config(tr.storage, 1, -1)
            res["storages"][stg]["default"] = lib.bp_table_kernel_config(
                table.handle, tr.storage, 1)
            # the library's own choice (a staged shape, or the direct kernel
            # where no shape holds the table's windows), timed the same way
            table.beamform_max(tr, 0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(2):
                table.beamform_max(tr, 0)
            e1.record()
            torch.cuda.synchronize()
            res["storages"][stg]["default_ms"] = e0.elapsed_time(e1) / 2
            del tr
        out["tables"][name] = res
        table.close()
    out["clocks"] = sampler.stop()
    print(json.dumps({"workload": "shapes", "n_gpus": 1, "data": "synthetic", **out}),
          flush=True)


# ----------------------------------------------------------------------------
# The stages either side of the beamformer (single GPU)
# ----------------------------------------------------------------------------

def run_stages(args, local_rank):
    """The tutorial's steps before and after beamform_max, each at its
    tutorial scale, device time (CUDA events) against the CPU code it
    replaces:
      features  -- envelope features of the 60-station x 3-channel x 180,000
                   sample network, and raw waveforms to trace rows in one call;
      detection -- threshold (rms, 7,200 s windows) and peaks (60 s apart)
                   of a day-long 25 Hz beam series (2,160,000 samples);
      ingest    -- 400,000 x 60 x 2 travel times (s) to relative delays."""
    import torch
    from scipy import signal
    from oracle import detection as odet
    from oracle import features as ofeat
    from oracle import ingest as oing
    from beampower_b200 import detection as det
    from beampower_b200.features import envelope
    from beampower_b200.ingest import sec_to_samp
    from beampower_b200.tables import TravelTimeTable
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    hbm_peak = None
    if os.path.exists(MEASURED_PEAKS):
        with open(MEASURED_PEAKS) as fh:
            hbm_peak = json.load(fh).get("hbm_gbs")
    steps, warm = max(args.steps, 1), max(args.warmup, 3)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def gpu_ms(fn):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def roof(bytes_, ms):
        gbs = bytes_ / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": gbs / hbm_peak if hbm_peak else None,
                "algorithmic_bytes": bytes_, "of": "measured (MEASURED_PEAKS.json)"}

    rng = np.random.default_rng(0)
    out = {}
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    # ---- features ----
    S, C, T, P = 60, 3, 180000, 2
    w = torch.from_numpy(rng.standard_normal((S, C, T)).astype(np.float32)).to(dev)
    A = torch.ones((S, C, P), device=dev)
    ms_env = gpu_ms(lambda: envelope(w))
    D = torch.zeros((64, S, P), dtype=torch.int32, device=dev)
    table = TravelTimeTable(D, torch.ones((64, S), device=dev), device=dev)
    ms_rows = gpu_ms(lambda: table.traces_from_waveforms(w, A))
    table.close()
    wc = w[:2].cpu().numpy()
    t0 = time.perf_counter()
    ofeat.waveform_features(wc)
    cpu_env = (time.perf_counter() - t0) * (S / 2)
    n = S * C * T
    out["features"] = {
        "samples": n, "envelope_ms": ms_env, "waveforms_to_trace_rows_ms": ms_rows,
        "value": n / (ms_env * 1e-3), "unit": "samples/s",
        "roofline": roof(8.0 * n, ms_env),
        "cpu_baseline": {"value": n / cpu_env, "unit": "samples/s", "cores": 1, "kind": "port",
                         "seconds": cpu_env,
                         "sample": "tutorial envelope (SciPy) on 2 of 60 stations, scaled"}}
    del w
    # ---- detection ----
    fs = 25.0
    nd = int(24 * 3600 * fs)
    x = np.abs(rng.standard_normal(nd + 24)).astype(np.float32)
    x = np.convolve(x, np.ones(25, np.float32) / 25, mode="valid")[:nd].astype(np.float32)
    x[nd - 2864:] = 0.0
    Wn, dist = int(7200 * fs), int(60 * fs)
    noise = rng.standard_normal(2864).astype(np.float32)
    xt = torch.from_numpy(x).to(dev)
    nt = torch.from_numpy(noise).to(dev)
    ms_thr = gpu_ms(lambda: det.time_dependent_threshold(xt, Wn, 0.66, "rms", 8.0,
                                                         white_noise=nt))
    thr = det.time_dependent_threshold(xt, Wn, 0.66, "rms", 8.0, white_noise=nt)
    ms_det = gpu_ms(lambda: det.detect(xt, threshold=thr, distance=dist))
    t0 = time.perf_counter()
    thr_c = odet.time_dependent_threshold(x, Wn, 0.66, "rms", 8.0, noise)
    t1 = time.perf_counter()
    pk = signal.find_peaks(x, distance=dist)[0]
    pk = pk[x[pk] > thr_c[pk]]
    t2 = time.perf_counter()
    out["detection"] = {
        "samples": nd, "threshold_ms": ms_thr, "detect_ms": ms_det,
        "value": nd / ((ms_thr + ms_det) * 1e-3), "unit": "samples/s",
        "detections": int(pk.size),
        "roofline": roof(16.0 * nd, ms_thr + ms_det),
        "note": "host-synchronised rounds (counts read back): latency bound, not HBM bound",
        "cpu_baseline": {"value": nd / (t2 - t0), "unit": "samples/s", "cores": 1,
                         "kind": "port", "seconds": t2 - t0, "threshold_s": t1 - t0,
                         "sample": "the whole series: tutorial threshold (NumPy) + "
                                   "scipy.signal.find_peaks"}}
    # ---- ingest ----
    tt = rng.uniform(0.0, 40.0, size=(400000, 60, 2)).astype(np.float32)
    ttd = torch.from_numpy(tt).to(dev)
    ms_ing = gpu_ms(lambda: sec_to_samp(ttd, 50.0, relative=True))
    t0 = time.perf_counter()
    oing.sec_to_samp(tt, 50.0, relative=True)
    cpu_ing = time.perf_counter() - t0
    ni = tt.size
    out["ingest"] = {
        "values": ni, "ms": ms_ing, "value": ni / (ms_ing * 1e-3), "unit": "delays/s",
        "roofline": roof(8.0 * ni, ms_ing),
        "cpu_baseline": {"value": ni / cpu_ing, "unit": "delays/s", "cores": 1, "kind": "port",
                         "seconds": cpu_ing, "sample": "the whole grid (NumPy)"}}
    # ---- the tutorial end to end (4,000 sources x 20 stations x 6,000 samples) ----
    out["pipeline"] = _pipeline_stage(dev, gpu_ms)
    out["pipeline_large"] = _pipeline_large(dev)
    clocks = sampler.stop()
    print(json.dumps({"workload": "stages", "n_gpus": 1, "steps": steps, "warmup": warm,
                      "data": "synthetic", "stages": out, "clocks": clocks}), flush=True)


def _pipeline_large(dev):
    """The tutorial end to end at the scale of the 400,000-source network:
    raw waveforms (60 x 3 x 180,000) and travel times in seconds
    (400,000 x 60 x 2) to detections, one call; GPU time only (the CPU
    reference's beamforming alone would take about ten minutes here, see the
    main benchmark's cpu_baseline)."""
    import torch
    from beampower_b200.pipeline import detect_events
    wl = make_workload(LARGE)
    fs = LARGE.fs
    D, W, A = wl["time_delays"], wl["weights_sources"], wl["weights_phases"]
    rng = np.random.default_rng(9)
    F = wl["waveform_features"]
    raw = torch.from_numpy((rng.standard_normal(F.shape) * (1.0 + F)).astype(np.float32)).to(dev)
    tt = torch.from_numpy((D / fs).astype(np.float32)).to(dev)
    kw = dict(window_duration_sec=600.0, num_dev=8.0, min_detection_interval_sec=60.0)
    detect_events(raw, tt, fs, A, W, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ev = detect_events(raw, tt, fs, A, W, **kw)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    N, S, P = D.shape
    return {"workload": LARGE.name + ", raw waveforms + travel times (s) -> detections",
            "ms": ms, "detections": int(ev.peaks.numel()),
            "beam_terms_per_s": nominal_terms(N, F.shape[2], S, P) / (ms * 1e-3),
            "note": "one call: travel-time conversion, table build, envelope features, "
                    "prestack, beamform_max, threshold, detections"}


def _pipeline_stage(dev, gpu_ms):
    """Raw waveforms and travel times (s) to detections: the tutorial's steps
    on the GPU (beampower_b200.pipeline.detect_events) against the same steps
    on the CPU -- SciPy envelopes, NumPy sec_to_samp, the reference's own C
    beamform_max (all host threads), NumPy threshold, SciPy find_peaks."""
    import torch
    from scipy import signal
    from oracle import detection as odet
    from oracle import features as ofeat
    from oracle import ingest as oing
    from oracle.oracle import Reference
    from beampower_b200.pipeline import detect_events
    from beampower_b200.synthetic import SMALL
    wl = make_workload(SMALL)
    fs = 25.0
    D, W, A = wl["time_delays"], wl["weights_sources"], wl["weights_phases"]
    rng = np.random.default_rng(8)
    F = wl["waveform_features"]
    raw = (rng.standard_normal(F.shape) * (1.0 + F)).astype(np.float32)
    tt = (D / fs).astype(np.float32)
    kw = dict(window_duration_sec=40.0, num_dev=3.0, min_detection_interval_sec=4.0)
    raw_d = torch.from_numpy(raw).to(dev)
    tt_d = torch.from_numpy(tt).to(dev)
    ms = gpu_ms(lambda: detect_events(raw_d, tt_d, fs, A, W, **kw))
    ev = detect_events(raw_d, tt_d, fs, A, W, **kw)
    ref = Reference()
    t0 = time.perf_counter()
    feats = ofeat.waveform_features(raw)
    delays = oing.sec_to_samp(tt, fs)
    U = ref.prestack(feats, A)
    bm, am = ref.beamform_max(U, delays, W, 0)
    zeros = int((bm == 0).sum())
    thr = odet.time_dependent_threshold(bm, int(40.0 * fs), 0.66, "rms", 3.0,
                                        rng.standard_normal(zeros).astype(np.float32))
    pk = signal.find_peaks(bm, distance=int(4.0 * fs))[0]
    pk = pk[bm[pk] > thr[pk]]
    cpu_s = time.perf_counter() - t0
    return {"workload": "small-4k-src-20-sta-6000-samples, raw waveforms + travel times (s)",
            "ms": ms, "detections": int(ev.peaks.numel()), "cpu_detections": int(pk.size),
            "cpu_baseline": {"seconds": cpu_s, "kind": "reference",
                             "cores": os.cpu_count(),
                             "sample": "the whole call: SciPy envelopes, NumPy sec_to_samp, "
                                       "reference C beamform_max, NumPy threshold, SciPy peaks"},
            "speedup": cpu_s / (ms * 1e-3)}


def run_sharded(args, rank, world, local_rank):
    """The large workload with its 400,000 sources split over the ranks: each
    rank builds the table of its block, prestacks, beamforms, rebases its
    keys, and one NCCL max all-reduce (8 T bytes) merges them; every rank
    decodes the result.  value = the whole workload's terms / the slowest
    rank's step (strong scaling)."""
    import torch
    from beampower_b200.core import check, load_library
    from beampower_b200.distributed import decode_shared, merge_keys, shard_range
    from beampower_b200.tables import TravelTimeTable, _stream_ptr
    dist_on = world > 1
    if dist_on:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = load_library("gpu")
    oob = 0 if args.out_of_bounds == "strict" else 1
    wl = make_workload(LARGE)
    F, A, D, W = (wl["waveform_features"], wl["weights_phases"], wl["time_delays"],
                  wl["weights_sources"])
    S, C, T = F.shape
    N, _, P = D.shape
    lo, hi = shard_range(N, rank, world)
    terms = nominal_terms(N, T, S, P)
    dF, dA = torch.from_numpy(F).to(dev), torch.from_numpy(A).to(dev)
    dD = torch.from_numpy(np.ascontiguousarray(D[lo:hi])).to(dev)
    dW = torch.from_numpy(np.ascontiguousarray(W[lo:hi])).to(dev)
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step(tables):
        table = TravelTimeTable(dD, dW, device=dev)
        traces = table.traces_from_features(dF, dA, storage=args.storage)
        bm = torch.zeros(T, dtype=torch.float32, device=dev)
        am = torch.zeros(T, dtype=torch.int32, device=dev)
        keys = torch.zeros(T, dtype=torch.int64, device=dev)
        table.beamform_max(traces, oob, out=(bm, am, keys))
        check(lib.bp_keys_to_shared_dev(keys.data_ptr(), T, lo, _stream_ptr()))
        merge_keys(keys)
        tables.append(table)
        return decode_shared(keys, dev)

    tables = []
    for _ in range(max(args.warmup, 3)):
        step(tables)
    torch.cuda.synchronize()
    for t in tables:
        t.close()
    tables = []
    launches0 = lib.bp_launch_count()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    barrier(dev)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.5)
    e0, e1 = ev(), ev()
    e0.record(stream)
    for _ in range(args.steps):
        bm, am = step(tables)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    launches = lib.bp_launch_count() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1), dev) / args.steps
    for t in tables:
        t.close()
    if rank == 0:
        print(json.dumps({
            "metric": "beam terms/s (src x t x sta x phase)", "value": terms / (ms * 1e-3),
            "unit": "beam terms/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.storage == "fp32" else args.storage, "data": "synthetic",
            "config": {"workload": LARGE.name, "n_sources": N, "n_stations": S,
                       "n_phases": P, "n_samples": T, "reduce": "max",
                       "out_of_bounds": args.out_of_bounds, "storage": args.storage,
                       "parallelism": f"sources split over {world} ranks",
                       "exchange": "NCCL int64 max all-reduce of 8 T bytes per call",
                       "l2": "inputs 418 MB > L2, no flush"},
            "clocks": clocks, "gpu_launches": launches}), flush=True)
    if dist_on:
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
