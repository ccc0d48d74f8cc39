"""The staged kernel's shared-memory carve keeps every field aligned for its
widest access (built and run on the host with nvcc; no GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_staged_smem_fields_aligned(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = tmp_path / "smem_layout_check"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-w",
                    "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "beampower_b200", "csrc"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "smem_layout_check.cu")],
                   check=True, capture_output=True, timeout=300)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout
