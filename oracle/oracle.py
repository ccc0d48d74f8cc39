"""ctypes front-end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py import this
module, as the checker or as the timed CPU baseline.  The beampower_b200
package never does.

Three CPU implementations are reachable from here:

* ``Oracle``    -- our C restatement, oracle/beamform_oracle.c;
* ``Reference`` -- the reference's own C/OpenMP library, compiled from
  beampower/src/beamform.c into oracle/_ref/beamform_cpu.so by oracle/Makefile;
  its entry points and argument order are those of beampower/core.py:14-59;
* ``fp64_*``    -- pure numpy restatements in float64, for tolerance checks on
  small cases.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_bp.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_CPU_SO = os.path.join(REF_DIR, "beamform_cpu.so")
REF_GPU_SO = os.path.join(REF_DIR, "beamform_gpu.so")

_f32p = ct.POINTER(ct.c_float)
_i32p = ct.POINTER(ct.c_int)
_sz = ct.c_size_t


REFERENCE_ENV = "BEAMPOWER_REFERENCE"


def reference_checkout() -> str | None:
    """The reference checkout, when one is present: the directory named by the
    BEAMPOWER_REFERENCE environment variable, else a checkout named
    ``reference`` beside this repository; None when neither holds the
    reference's sources."""
    repo = os.path.dirname(HERE)
    for cand in (os.environ.get(REFERENCE_ENV),
                 os.path.join(os.path.dirname(repo), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "beampower", "src")):
            return cand
    return None


def build(reference_root: str | None = None) -> None:
    """Compile the oracle, and the reference libraries when `reference_root`
    (a reference checkout) holds the reference's sources."""
    targets = ["oracle"]
    args = []
    if reference_root and os.path.isdir(os.path.join(reference_root, "beampower", "src")):
        targets.append("ref")
        args.append(f"REF_ROOT={reference_root}")
    subprocess.run(["make", "-s", "-C", HERE, *args] + targets, check=True)


def _fp(a):
    return a.ctypes.data_as(_f32p)


def _ip(a):
    return a.ctypes.data_as(_i32p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """Our C restatement of the reference algorithm (see beamform_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise OSError(f"oracle library not built: {path} (run make -C oracle)")
        lib = ct.CDLL(path)
        lib.bpo_minmax.argtypes = [_i32p, _f32p, _sz, _sz, _sz, ct.c_int, _i32p]
        lib.bpo_prestack.argtypes = [_f32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int, _f32p]
        lib.bpo_beamform.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int,
                                     ct.c_int, _f32p]
        lib.bpo_beamform_max.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int,
                                         ct.c_int, _f32p, _i32p, _i32p]
        lib.bpo_beamform_differential.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz,
                                                  ct.c_int, _f32p]
        _i64p = ct.POINTER(ct.c_int64)
        lib.bpo_beamform_max_at.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int,
                                            ct.c_int, _i64p, _sz, _f32p, _i32p, _i32p]
        for f in (lib.bpo_minmax, lib.bpo_prestack, lib.bpo_beamform, lib.bpo_beamform_max,
                  lib.bpo_beamform_differential, lib.bpo_beamform_max_at):
            f.restype = None
        self.lib = lib

    def minmax(self, delays, weights, num_threads=0):
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        n, s, p = d.shape
        out = np.empty((n, 2), dtype=np.int32)
        self.lib.bpo_minmax(_ip(d), _fp(w), n, s, p, num_threads, _ip(out))
        return out

    def prestack(self, features, weights_phases, num_threads=0):
        f = _c(features, np.float32)
        a = _c(weights_phases, np.float32)
        s, c, t = f.shape
        p = a.shape[2]
        out = np.empty((s, t, p), dtype=np.float32)
        self.lib.bpo_prestack(_fp(f), _fp(a), t, s, c, p, num_threads, _fp(out))
        return out

    def beamform(self, prestacked, delays, weights, out_of_bounds=0, num_threads=0,
                 out=None):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        beam = np.zeros((n, t), dtype=np.float32) if out is None else out
        self.lib.bpo_beamform(_fp(u), _ip(d), _fp(w), t, n, s, p, int(out_of_bounds),
                              num_threads, _fp(beam))
        return beam

    def beamform_max(self, prestacked, delays, weights, out_of_bounds=0, num_threads=0):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        bm = np.zeros(t, dtype=np.float32)
        am = np.zeros(t, dtype=np.int32)
        mm = np.empty((max(n, 1), 2), dtype=np.int32)
        self.lib.bpo_beamform_max(_fp(u), _ip(d), _fp(w), t, n, s, p, int(out_of_bounds),
                                  num_threads, _fp(bm), _ip(am), _ip(mm))
        return bm, am

    def beamform_max_at(self, prestacked, delays, weights, times, out_of_bounds=0,
                        num_threads=0):
        """(beam_max, argmax) at the given sample indexes only; beam_max is 0
        where no source is a candidate."""
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        tt = _c(times, np.int64)
        s, t, p = u.shape
        n = d.shape[0]
        bm = np.zeros(len(tt), dtype=np.float32)
        am = np.zeros(len(tt), dtype=np.int32)
        mm = np.empty((max(n, 1), 2), dtype=np.int32)
        self.lib.bpo_beamform_max_at(_fp(u), _ip(d), _fp(w), t, n, s, p, int(out_of_bounds),
                                     num_threads, tt.ctypes.data_as(ct.POINTER(ct.c_int64)),
                                     len(tt), _fp(bm), _ip(am), _ip(mm))
        return bm, am

    def beamform_differential(self, prestacked, delays, weights, num_threads=0):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        beam = np.zeros(n, dtype=np.float32)
        self.lib.bpo_beamform_differential(_fp(u), _ip(d), _fp(w), t, n, s, p, num_threads,
                                           _fp(beam))
        return beam


class Reference:
    """The reference's own CPU library, argtypes of beampower/core.py:14-59.

    Note the reference's prestack prototype names its first size argument
    n_sources; the value passed is the number of samples (beampower.py:279).
    """

    def __init__(self, path: str = REF_CPU_SO):
        if not os.path.exists(path):
            raise OSError(f"reference library not built: {path} (run make -C oracle ref)")
        lib = ct.CDLL(path)
        lib.beamform.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int, ct.c_int,
                                 _f32p]
        lib.beamform_max.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int,
                                     ct.c_int, _f32p, _i32p]
        lib.prestack_waveform_features.argtypes = [_f32p, _f32p, _sz, _sz, _sz, _sz, ct.c_int,
                                                   _f32p]
        lib.beamform_differential.argtypes = [_f32p, _i32p, _f32p, _sz, _sz, _sz, _sz,
                                              ct.c_int, _f32p]
        for f in (lib.beamform, lib.beamform_max, lib.prestack_waveform_features,
                  lib.beamform_differential):
            f.restype = None
        self.lib = lib

    def prestack(self, features, weights_phases, num_threads=-1):
        f = _c(features, np.float32)
        a = _c(weights_phases, np.float32)
        s, c, t = f.shape
        p = a.shape[2]
        out = np.zeros((s, t, p), dtype=np.float32)
        self.lib.prestack_waveform_features(_fp(f), _fp(a), t, s, c, p, int(num_threads),
                                            _fp(out))
        return out

    def beamform(self, prestacked, delays, weights, out_of_bounds=0, num_threads=-1):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        beam = np.zeros((n, t), dtype=np.float32)
        self.lib.beamform(_fp(u), _ip(d), _fp(w), t, n, s, p, int(out_of_bounds),
                          int(num_threads), _fp(beam))
        return beam

    def beamform_max(self, prestacked, delays, weights, out_of_bounds=0, num_threads=-1):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        bm = np.zeros(t, dtype=np.float32)
        am = np.zeros(t, dtype=np.int32)
        self.lib.beamform_max(_fp(u), _ip(d), _fp(w), t, n, s, p, int(out_of_bounds),
                              int(num_threads), _fp(bm), _ip(am))
        return bm, am

    def beamform_differential(self, prestacked, delays, weights, num_threads=-1):
        u = _c(prestacked, np.float32)
        d = _c(delays, np.int32)
        w = _c(weights, np.float32)
        s, t, p = u.shape
        n = d.shape[0]
        beam = np.zeros(n, dtype=np.float32)
        self.lib.beamform_differential(_fp(u), _ip(d), _fp(w), t, n, s, p, int(num_threads),
                                       _fp(beam))
        return beam


# ----------------------------------------------------------------------------
# float64 numpy restatements (small cases only)
# ----------------------------------------------------------------------------

def fp64_prestack(features, weights_phases):
    """U[s, t, p] = sum_c alpha[s, c, p] F[s, c, t] in float64
    (beamform.c:108-152)."""
    f = np.asarray(features, dtype=np.float64)
    a = np.asarray(weights_phases, dtype=np.float64)
    return np.einsum("sct,scp->stp", f, a)


def fp64_minmax(delays, weights):
    """Per-source (min, max) delay over weighted stations; sources without a
    weighted station get (INT_MAX, INT_MIN) (beamform.c:10-47)."""
    d = np.asarray(delays, dtype=np.int64)
    w = np.asarray(weights)
    m = (w != 0)[:, :, None]
    lo = np.where(m, d, np.iinfo(np.int32).max).min(axis=(1, 2))
    hi = np.where(m, d, np.iinfo(np.int32).min).max(axis=(1, 2))
    return np.stack([lo, hi], axis=1).astype(np.int32)


def fp64_beams(prestacked, delays, weights, out_of_bounds=0):
    """Full (N, T) float64 beam plus the (N, T) validity mask of the rule in
    beamform_oracle.c (strict: whole network in bounds; flexible: always)."""
    u = np.asarray(prestacked, dtype=np.float64)
    d = np.asarray(delays, dtype=np.int64)
    w = np.asarray(weights, dtype=np.float64)
    s_n, t_n, p_n = u.shape
    n = d.shape[0]
    t = np.arange(t_n)
    beam = np.zeros((n, t_n))
    for s in range(s_n):
        for p in range(p_n):
            idx = t[None, :] + d[:, s, p][:, None]
            ok = (idx >= 0) & (idx < t_n)
            vals = np.where(ok, u[s, np.clip(idx, 0, t_n - 1), p], 0.0)
            ws = w[:, s][:, None]
            beam += np.where(ws != 0, ws * vals, 0.0)
    mm = fp64_minmax(delays, weights).astype(np.int64)
    if out_of_bounds == 0:
        has = mm[:, 0] <= mm[:, 1]
        valid = has[:, None] & (t[None, :] + mm[:, :1] >= 0) & (t[None, :] + mm[:, 1:] < t_n)
    else:
        valid = np.ones((n, t_n), dtype=bool)
    return beam, valid
