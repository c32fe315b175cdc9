"""Build recipe of the product: libstormgpu.so (CUDA kernels + C ABI, sm_100a only) and the
storm-nucleotide / storm-color command-line binaries linked against it.  Outputs stay in the
source tree (storm_b200/lib, storm_b200/bin) so that they travel with the repository."""
from __future__ import annotations

import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
BIN_DIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIB_DIR, "libstormgpu.so")
HOST_LIB = os.path.join(LIB_DIR, "libstormhost.so")
CU_SOURCES = ["stormgpu.cu", "index_build.cu", "map_kernels.cu", "sw_filter.cu", "gather.cu", "intpeak.cu", "align_noalloc.cu", "server.cu", "genome_map.cu", "genome_map_ctx.cu", "autotune.cu"]
HOST_SOURCES = ["host/storm_host.c", "host/storm_cli.c", "host/storm_gpu_main.c"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for root, _, files in os.walk(CSRC):
        out += [os.path.join(root, f) for f in files if f.endswith((".cu", ".cuh", ".c", ".h"))]
    out.append(os.path.join(os.path.dirname(PKG), "include", "stormgpu.h"))
    return out


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    deps = _deps()
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    if force or _stale(LIB, deps):
        objs = []
        for src in CU_SOURCES:
            obj = os.path.join(objdir, src.replace(".cu", ".o"))
            if force or _stale(obj, deps):
                _run([nvcc()] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj], verbose)
            objs.append(obj)
        _run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + ["-cudart", "static"], verbose)
    if force or _stale(HOST_LIB, deps):
        _run(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-fPIC", "-shared", "-o", HOST_LIB,
              os.path.join(CSRC, "host", "storm_host.c"), "-lm"], verbose)
    for colour, name in ((0, "storm-nucleotide"), (1, "storm-color")):
        exe = os.path.join(BIN_DIR, name)
        if force or _stale(exe, deps + [LIB]):
            _run(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-DSTORM_COLOUR=%d" % colour, "-o", exe]
                 + [os.path.join(CSRC, s) for s in HOST_SOURCES]
                 + ["-L" + LIB_DIR, "-lstormgpu", "-Wl,-rpath,$ORIGIN/../lib", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
