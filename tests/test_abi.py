"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; the ctypes table binds them all; front-end argument
errors behave like the reference's (no GPU work involved)."""
import ctypes as ct
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"BP_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_drop_ins():
    names = declared_symbols()
    for sym in ("beamform", "beamform_max", "prestack_waveform_features",
                "beamform_differential", "bp_beamform_max_dev", "bp_table_create"):
        assert sym in names


def test_library_exports_every_declared_symbol():
    from beampower_b200.core import LIBRARIES
    path = LIBRARIES["gpu"]["filepath_library"]
    assert os.path.exists(path), "build the library first (python -m beampower_b200.build)"
    lib = ct.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_table_covers_header():
    from beampower_b200.core import SIGNATURES, load_library
    assert set(declared_symbols()) <= set(SIGNATURES)
    lib = load_library("gpu")
    assert lib.bp_version().startswith(b"beampower_b200")


def test_integration_guide_lists_every_symbol():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert [s for s in declared_symbols() if f"`{s}`" not in text] == []


def test_reference_argtypes_kept():
    """The drop-in argtypes equal beampower/core.py:65-87 (restype added)."""
    from beampower_b200.core import LIBRARIES
    f32p, i32p = ct.POINTER(ct.c_float), ct.POINTER(ct.c_int)
    assert LIBRARIES["gpu"]["beamform_argtypes"] == [
        f32p, i32p, f32p, ct.c_size_t, ct.c_size_t, ct.c_size_t, ct.c_size_t, ct.c_int, f32p]
    assert LIBRARIES["gpu"]["beamform_max_argtypes"] == [
        f32p, i32p, f32p, ct.c_size_t, ct.c_size_t, ct.c_size_t, ct.c_size_t, ct.c_int, f32p,
        i32p]


def test_argument_errors_without_gpu():
    """Invalid sizes are rejected before any CUDA call, with a message."""
    from beampower_b200.core import load_library
    lib = load_library("gpu")
    rc = lib.bp_beamform_host(None, None, None, None, 10, 10, 0, 3, 2, 0, 1, 0, None, None, None)
    assert rc == 1 and b"n_stations" in lib.bp_last_error()
    rc = lib.bp_beamform_host(None, None, None, None, 10, 10, 4, 3, 2, 7, 1, 0, None, None, None)
    assert rc == 1 and b"out_of_bounds" in lib.bp_last_error()


def test_frontend_error_behaviour(capsys):
    import beampower_b200 as bp
    F = np.zeros((2, 3, 10), np.float32)
    D = np.zeros((4, 2, 2), np.int32)
    A = np.zeros((2, 3, 2), np.float32)
    W = np.ones((4, 2), np.float32)
    assert bp.beamform(F, D, A, W, out_of_bounds="loose") is None
    assert "out_of_bounds should be" in capsys.readouterr().out
    assert bp.beamform(F, D, A, W, mode="sideways") == 1
    assert "Mode should either be" in capsys.readouterr().out
    assert bp.beamform(F, D, A, W, reduce="mean") == 1      # the reference's fall-through
    with pytest.raises(NameError):
        bp.beamform(F, D, A, W, device="cpu")
    with pytest.raises(NameError):
        bp.load_library("tpu")


def test_frontend_draws_from_numpy_like_the_reference(capsys):
    """beampower.py:113-114 draws once from NumPy's global generator per call
    that passes the out_of_bounds check, whatever the mode; a seeded caller's
    later draws stay where they were with the drop-in."""
    import beampower_b200 as bp
    F = np.zeros((2, 3, 10), np.float32)
    D = np.zeros((4, 2, 2), np.int32)
    A = np.zeros((2, 3, 2), np.float32)
    W = np.ones((4, 2), np.float32)
    np.random.seed(1234)
    want = np.random.random(3)
    np.random.seed(1234)
    assert bp.beamform(F, D, A, W, mode="sideways") == 1   # one draw
    assert bp.beamform(F, D, A, W, out_of_bounds="loose") is None  # none
    assert bp.beamform(F, D, A, W, reduce="mean") == 1     # one draw
    assert np.random.random() == want[2]
    capsys.readouterr()


def test_key_order_matches_reference_max_rule():
    """Host restatement of the packed key: order = (value, -index), NaN and
    values <= -FLT_MAX are not candidates, decode inverts encode."""
    import struct
    fmax = np.finfo(np.float32).max

    def ordered(v):
        b = struct.unpack("<I", struct.pack("<f", v))[0]
        if b == 0x80000000:
            b = 0
        return (~b & 0xFFFFFFFF) if b & 0x80000000 else (b | 0x80000000)

    def key(v, i):
        if not (v > -fmax):
            return 0
        return (ordered(v) << 32) | (0xFFFFFFFF - i)

    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.standard_normal(200).astype(np.float32) * 1e3,
                           np.float32([0.0, -0.0, np.inf, -np.inf, np.nan, fmax, -fmax,
                                       1e-42, -1e-42])])
    for _ in range(200):
        idx = rng.choice(len(vals), size=6)
        cand = [(float(np.float32(vals[i])), j) for j, i in enumerate(idx)]
        best, besti = -fmax, 0
        for v, j in cand:
            if v > best:
                best, besti = v, j
        k = max(key(v, j) for v, j in cand)
        if best > -fmax:
            assert k != 0 and 0xFFFFFFFF - (k & 0xFFFFFFFF) == besti
        else:
            assert k == 0


def test_kernel_configs_described():
    from beampower_b200.autotune import configs
    cfgs = configs()
    assert len(cfgs) >= 6
    for c, d in cfgs:
        # one block per 64-source table tile, or blocks sharing a tile
        assert d["sources_per_thread"] * d["consumer_warps"] == d["sources_per_block"]
        assert 64 % d["sources_per_block"] == 0
        assert d["samples_per_lane"] % 2 == 0 and d["stages"] >= 2
        assert d["stations_per_stage"] in (1, 2) and d["blocks_per_sm"] >= 1


def test_every_package_module_imports():
    """Every module of the package imports on a machine without a GPU (the
    GPU-only tests would otherwise be the first to see a syntax error)."""
    import importlib
    import pkgutil
    import beampower_b200
    names = [m.name for m in pkgutil.iter_modules(beampower_b200.__path__)]
    assert "stream" in names and "batch" in names
    for name in names:
        importlib.import_module(f"beampower_b200.{name}")


def test_noalloc_refusal_recorded_without_gpu():
    """The allocation-free entry point refuses sizes beyond its fixed array
    before any CUDA call, and records the reason for bp_last_error()."""
    import beampower_b200 as bp
    lib = bp.load_library("gpu")
    assert lib.bp_beamform_max_noalloc(None, 524288 + 1, 0, 524288 + 1, None, None, 10, 2, 2,
                                       0, None, None, None) == 6  # BP_ERR_SCRATCH_LIMIT
    msg = lib.bp_last_error()
    assert b"scratch" in msg and b"524288" in msg
    assert lib.bp_beamform_max_noalloc(None, 100, 0, 100, None, None, 10, 2, 2, 7,
                                       None, None, None) == 1  # BP_ERR_INVALID_ARGUMENT
    assert b"out_of_bounds" in lib.bp_last_error()


def test_cmake_project_configures(tmp_path):
    """The CMake target (CMakeLists.txt, sm_100a) configures: a CUDA
    compiler, the toolkit's cuFFT and every source under csrc/ are found.
    Building it takes minutes and is not part of this suite."""
    import shutil
    import subprocess
    cmake = shutil.which("cmake")
    if cmake is None:
        pytest.skip("cmake is not installed")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([cmake, "-S", root, "-B", str(tmp_path)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert (tmp_path / "CMakeCache.txt").exists()


def _c_kind(decl):
    """Kind of a C parameter / return declaration: ptr, u64, i64, i32, f32, f64."""
    d = decl.replace("const", " ").strip()
    if "*" in d:
        return "ptr"
    base = " ".join(d.split()[:-1]) if len(d.split()) > 1 and d.split()[-1] not in (
        "int", "float", "double", "size_t") else d
    base = " ".join(base.split())
    return {"size_t": "u64", "uint64_t": "u64", "unsigned long long": "u64",
            "int64_t": "i64", "long long": "i64", "int": "i32", "int32_t": "i32",
            "float": "f32", "double": "f64"}[base]


def _ctypes_kind(t):
    if t is None:
        return None
    if issubclass(t, (ct._Pointer, ct.c_void_p, ct.c_char_p)):
        return "ptr"
    if t in (ct.c_float, ct.c_double):
        return "f32" if t is ct.c_float else "f64"
    signed = t(-1).value == -1
    return {(8, False): "u64", (8, True): "i64", (4, True): "i32"}[(ct.sizeof(t), signed)]


def test_ctypes_signatures_match_header_prototypes():
    """Every SIGNATURES entry has the header prototype's argument count and
    the same kind (pointer, 32/64-bit integer, float, double) per argument
    and for the result, so a drifted table cannot pass arguments silently."""
    from beampower_b200.core import SIGNATURES
    text = "\n".join(open(h).read() for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = re.findall(r"BP_API\s+([\w\s\*]+?)\b(\w+)\s*\(([^)]*)\)\s*;", text)
    assert len(protos) == len(declared_symbols())
    for ret, name, params in protos:
        args = [p for p in (x.strip() for x in params.split(",")) if p and p != "void"]
        argtypes, restype = SIGNATURES[name]
        assert len(args) == len(argtypes), name
        for i, (a, t) in enumerate(zip(args, argtypes)):
            assert _c_kind(a) == _ctypes_kind(t), f"{name} argument {i}: {a}"
        assert _c_kind(ret + " r") == _ctypes_kind(restype), f"{name} result"


def test_struct_mirrors_match_header_layout(tmp_path):
    """The ctypes mirrors of bp_table_info, bp_record and bp_peak_options have
    the header structs' size and every field at the header's offset: a C
    program built from the header by gcc prints them."""
    import shutil
    import subprocess
    from beampower_b200.core import PeakOptions, Record, TableInfo
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.skip("no C compiler")
    mirrors = {"bp_table_info": TableInfo, "bp_record": Record, "bp_peak_options": PeakOptions}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "beampower_b200.h"',
             "int main(void) {"]
    for cname, st in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in st._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {(a, b): int(c) for a, b, c in (ln.split() for ln in out.splitlines())}
    for cname, st in mirrors.items():
        assert got[(cname, "size")] == ct.sizeof(st), cname
        for field, _ in st._fields_:
            assert got[(cname, field)] == getattr(st, field).offset, f"{cname}.{field}"
