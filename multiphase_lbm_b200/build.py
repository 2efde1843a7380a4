"""Build recipe for the native parts of multiphase_lbm_b200.

* ``libmlbm.so``  -- the CUDA kernels (sm_100a) and the C ABI of
  ``include/mlbm.h`` / ``include/mlbm_compat.h``, plus the host driver
  (command-file parser, geometry, statistics, VTK output).
* ``mlbm``        -- the command-line program, a drop-in for the reference's
  ``multiphaselbm <commandFile>`` (src/main.cc).

Built in-tree with nvcc for ``sm_100a`` only; ``python -m
multiphase_lbm_b200.build`` or ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmlbm.so")
EXE = os.path.join(PKG, "mlbm")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
           "-Xcompiler", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC]

CXX = "/usr/bin/g++"
# Host code: no FMA contraction, so the voxeliser and the statistics round
# exactly as the reference's host code does.
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
            "-Wall", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
            "-I", "/usr/local/cuda/include"]

CUDA_SOURCES = ["capi.cu", "compat.cu", "noalloc.cu",
                "batch.cu", "compact.cu", "packing.cu", "clusters_gpu.cu",
                "slab.cu", "checkpoint.cu"]
HOST_SOURCES = ["host/driver.cpp", "host/geometry.cpp", "host/output.cpp",
                "host/clusters.cpp"]
CLI_SOURCE = "host/main.cpp"


def _sources():
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES + HOST_SOURCES]
    return [s for s in srcs if os.path.exists(s)]


def _deps():
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files
                if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    out += [os.path.join(ROOT, "include", f)
            for f in os.listdir(os.path.join(ROOT, "include"))]
    out.append(os.path.abspath(__file__))
    return out


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libmlbm.so (and the mlbm CLI) in-tree; returns the library path."""
    if force or _stale(LIB):
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        procs = []
        for src in _sources():
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            if src.endswith(".cu"):
                cmd = [NVCC, *ARCH, *NVFLAGS, "-c", src, "-o", obj]
            else:
                cmd = [CXX, *CXXFLAGS, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd)))
            objs.append(obj)
        for src, p in procs:
            if p.wait() != 0:
                raise RuntimeError(f"nvcc failed on {src}")
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", *objs,
               "-o", LIB, "-lcuda"]
        subprocess.run(cmd, check=True)
        cli = os.path.join(CSRC, CLI_SOURCE)
        if os.path.exists(cli):
            cmd = [CXX, *CXXFLAGS, cli, "-o", EXE, "-L", PKG, "-lmlbm",
                   "-Wl,-rpath,$ORIGIN"]
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
