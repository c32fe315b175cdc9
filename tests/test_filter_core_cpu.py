"""The packed 16-bit filter core of the CUDA kernel (storm_b200/csrc/filter_core.cuh), compiled
for the host, against the oracle's filter on random cases (widths 2-16, short and long reads,
varied scores and thresholds, windows before, inside and after the sequence)."""
import os
import shutil
import subprocess

import pytest

import ffi

NVCC = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else shutil.which("nvcc")


@pytest.mark.skipif(NVCC is None, reason="nvcc not available")
def test_filter_core_matches_oracle(tmp_path):
    ffi.ensure_built()
    exe = str(tmp_path / "fch")
    src = os.path.join(os.path.dirname(__file__), "filter_core_host.cu")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", src, "-o", exe,
                    "-L" + ffi.ORACLE_DIR, "-loracle", "-Xlinker", "-rpath=" + ffi.ORACLE_DIR], check=True)
    p = subprocess.run([exe, "60000"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "checked 60000" in p.stdout
