"""Autotuner of the staged kernel's shape.

The library compiles the staged kernel in several shapes (sources per
thread, samples per lane, consumer warps, ring stages, stations per ring
stage, sources per block; see ``bp_kernel_config_describe`` and
``bp_kernel_config_shape``), all over the same 64-source tables.  Which is
fastest depends on the storage type (FP32 is shared-memory bound, 16-bit
storage issue bound), the number of phases and the tables' delay spread.
``autotune`` times every shape on the caller's own table and traces, keeps
the fastest for that (storage, reduce) in the process, and records it in a
JSON cache keyed by GPU, storage, reduce, stations, phases and a delay-spread
class; ``apply_cached`` restores the choices in a later process.
"""
from __future__ import annotations

import ctypes as ct
import json
import os

from .core import REDUCE_MAX, REDUCE_NONE, STORAGE, check, load_library

CACHE_ENV = "BEAMPOWER_B200_AUTOTUNE_CACHE"


def cache_path():
    return os.environ.get(CACHE_ENV) or os.path.join(
        os.path.expanduser("~"), ".cache", "beampower_b200", "autotune.json")


def configs():
    """[(id, {sources_per_thread, samples_per_lane, consumer_warps, stages,
    stations_per_stage, sources_per_block, blocks_per_sm})]."""
    lib = load_library("gpu")
    out = []
    for c in range(lib.bp_kernel_config_count()):
        v = [ct.c_int() for _ in range(4)]
        check(lib.bp_kernel_config_describe(c, *[ct.byref(x) for x in v]))
        x = [ct.c_int() for _ in range(3)]
        check(lib.bp_kernel_config_shape(c, *[ct.byref(y) for y in x]))
        out.append((c, dict(zip(("sources_per_thread", "samples_per_lane", "consumer_warps",
                                 "stages", "stations_per_stage", "sources_per_block",
                                 "blocks_per_sm"), [y.value for y in v + x]))))
    return out


def _gpu_key():
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|{p.multi_processor_count}"


def _problem_key(table, storage, reduce):
    spread = table.info["max_spread"]
    spread_class = 0 if spread < 256 else (1 if spread < 1024 else 2)
    return (f"{_gpu_key()}|storage={storage}|reduce={reduce}|S={table.n_stations}"
            f"|P={table.n_phases}|spread={spread_class}")


def _load():
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(data):
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(table, traces, out_of_bounds=0, reduce="max", repeats=2, write_cache=True):
    """Time every kernel shape on (table, traces); select the fastest for the
    traces' storage and the given reduce.  Returns {config: ms} and the choice;
    shapes whose shared memory does not fit this table are None."""
    import torch
    lib = load_library("gpu")
    storage = traces.storage
    red = REDUCE_MAX if reduce == "max" else REDUCE_NONE
    prev = lib.bp_get_kernel_config(storage, red)
    times = {}
    for c, _ in configs():
        check(lib.bp_set_kernel_config(storage, red, c))
        if lib.bp_table_kernel_config(table.handle, storage, red) != c:
            times[c] = None  # does not fit this table (another shape would run)
            continue
        run = (lambda: table.beamform_max(traces, out_of_bounds)) if red == REDUCE_MAX else \
            (lambda: table.beamform(traces, out_of_bounds))
        run()  # warm-up (kernel attributes, lazy loading)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(repeats):
            run()
        ev1.record()
        torch.cuda.synchronize()
        times[c] = ev0.elapsed_time(ev1) / repeats
    ran = {c: t for c, t in times.items() if t is not None}
    if not ran:
        check(lib.bp_set_kernel_config(storage, red, prev))
        return {"times_ms": times, "best": None, "previous": prev}
    best = min(ran, key=ran.get)
    check(lib.bp_set_kernel_config(storage, red, best))
    if write_cache:
        data = _load()
        data[_problem_key(table, storage, reduce)] = {"config": best, "ms": times}
        _store(data)
    return {"times_ms": times, "best": best, "previous": prev}


def apply_cached(table=None, storage="fp32", reduce="max"):
    """Apply a cached choice for this GPU (and table class, when given)."""
    lib = load_library("gpu")
    st = STORAGE[storage] if isinstance(storage, str) else storage
    red = REDUCE_MAX if reduce == "max" else REDUCE_NONE
    data = _load()
    if table is not None:
        hit = data.get(_problem_key(table, st, reduce))
        if hit:
            check(lib.bp_set_kernel_config(st, red, int(hit["config"])))
            return int(hit["config"])
        return None
    prefix = f"{_gpu_key()}|storage={st}|reduce={reduce}|"
    for k, v in data.items():
        if k.startswith(prefix):
            check(lib.bp_set_kernel_config(st, red, int(v["config"])))
            return int(v["config"])
    return None
