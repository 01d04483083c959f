"""Build recipe for the in-tree CUDA library (sm_100a) and the oracle.

nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false ...
-fmad=false is part of the numerics contract: the kernels place every fused
multiply-add explicitly, so the compiler must not contract anything else.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpbf_b200.so")

SOURCES = ["pbf_kernels.cu", "pbf_pairs.cu", "pbf_mlp.cu", "pbf_capi.cu", "pbf_noalloc.cu", "pbf_render.cu"]
HEADERS = ["pbf_device.cuh", "pbf_kernels.h", "pbf_mlp.h", "pbf_mlp_dev.cuh", "pbf_tc.cuh", "pbf_packed.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(REPO, "include", "pbf.h")]
    if force or _stale(LIB, deps):
        cmd = [_nvcc()] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


def reference_dir() -> str:
    """Where the reference's source tree is on this machine, or "" when it is not:
    $PBF_REFERENCE_DIR, else the build container's read-only checkout. The
    reference is needed only to build the test checkers; a machine without it
    uses the checkers built where it was present."""
    for d in (os.environ.get("PBF_REFERENCE_DIR", ""), "/root/reference"):
        if d and os.path.isdir(os.path.join(d, "src")) and os.path.isdir(os.path.join(d, "kernels")):
            return d
    return ""


def build_oracle(verbose: bool = False) -> None:
    """Test infrastructure: the CPU restatement, plus the reference checkers (the
    reference's CPU and CUDA solvers built from its sources, and the test program
    that drives this library through the reference's own entry points) when the
    reference sources are present on this machine."""
    odir = os.path.join(REPO, "oracle")
    targets = ["oracle"]
    ref = reference_dir()
    args = ["make", "-s", "-C", odir]
    if ref:
        targets += ["refcpu", "refgpu", "refapp"]
        args.append(f"REF={ref}")
    subprocess.run(args + targets, check=True, stdout=None if verbose else subprocess.DEVNULL)


def build(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_oracle(verbose=verbose)


if __name__ == "__main__":
    build(force=True, verbose=True)
