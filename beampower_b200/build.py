"""Build libbeampower_b200.so for sm_100a with nvcc (in-tree, no JIT cache).

    python -m beampower_b200.build            # build if sources changed
    python -m beampower_b200.build --force    # always rebuild
    python -m beampower_b200.build --checked  # the index-checked variant
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libbeampower_b200.so")
# The same sources with the staged kernel's index checks compiled in
# (BP_DEBUG_CHECKS): load it with BEAMPOWER_B200_LIBRARY=<path>.
CHECKED_LIB = os.path.join(LIBDIR, "libbeampower_b200_checked.so")

COMPILE_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]
LINK_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-shared",
    "-cudart", "static",
    "-lcufft",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(INCLUDE, "*.h")) + [os.path.abspath(__file__)])


def up_to_date(lib=LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(p) <= t for p in _deps())


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _host_compiler():
    # nvcc's host compiler: the system gcc (the image's CC wrapper is incomplete)
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/gcc") else []


def build(force: bool = False, verbose: bool = False, extra=(), jobs=None,
          checked: bool = False) -> str:
    """Compile every .cu under csrc/ (one nvcc per file, in parallel) and link
    them into one shared library; return its path.  checked=True builds the
    index-checked variant (CHECKED_LIB) from the same sources."""
    lib = CHECKED_LIB if checked else LIB
    if checked:
        extra = (*extra, "-DBP_DEBUG_CHECKS=1")
    if not force and up_to_date(lib):
        return lib
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj_checked" if checked else "obj")
    os.makedirs(objdir, exist_ok=True)
    cc = _host_compiler()
    jobs = jobs or max(1, min(len(sources()), os.cpu_count() or 1))

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc(), *cc, *COMPILE_FLAGS, *extra, "-I", INCLUDE, "-I", CSRC, "-c", src,
               "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(compile_one, sources()))
    # objects of sources that no longer exist
    current = {obj for _s, obj, _r in results}
    for stale in glob.glob(os.path.join(objdir, "*.o")):
        if stale not in current:
            os.remove(stale)
    failed = False
    for src, _obj, r in results:
        if r.stdout or r.stderr:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {src}\n")
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc")
    tmp = lib + ".tmp"
    # cuFFT (envelope features) is found through the toolkit's lib64 at run time
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(
        nvcc() if os.path.sep in nvcc() else "/usr/local/cuda/bin/nvcc"))), "lib64")
    cmd = [nvcc(), *cc, *LINK_FLAGS, *(obj for _s, obj, _r in results),
           "-Xlinker", "-rpath=" + cuda_lib, "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    args = sys.argv[1:]
    ptxas = ["-Xptxas", "-v"] if "--ptxas-v" in args else []
    print(build(force="--force" in args or bool(ptxas), verbose=True, extra=ptxas,
                checked="--checked" in args))
