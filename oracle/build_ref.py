"""Build recipe for ``oracle/_ref``: the reference's own code compiled for the CPU.

Test infrastructure only (the oracle) -- nothing built here is shipped or
timed as the product.

The reference fixes the lattice size at compile time (``#define lx/ly/lz`` at
include/lbm_model.cuh:4-6).  For every size listed in ``SIZES`` this script
copies the reference's ``include/``, ``src/`` and ``external/`` into a scratch
directory under /tmp (the reference mount is read-only and no reference source
is ever copied into this repository), sets the three size macros in that copy,
and compiles with g++:

* ``oracle/_ref/libref_<lx>x<ly>x<lz>.so`` -- the reference kernels and device
  functions (include/iteration_kernel.cuh, include/iteration_device.cuh) plus
  the reference host driver (src/multiphase_lbm.cu), run on the host through
  oracle/ref_shim.h and oracle/ref_harness.cpp (OpenMP over x);
* ``oracle/_ref/multiphaselbm_cpu_<lx>x<ly>x<lz>`` -- the reference program
  (src/main.cc) linked against the same objects;
* ``oracle/_ref/ref_cuda_timer_200x200x200`` -- the reference's own CUDA
  time step, built for sm_100a and timed between CUDA events by
  oracle/ref_cuda_timer.cu (a reported baseline only).

Run: ``python oracle/build_ref.py [--sizes 16x12x10,64x64x64]``.  Without the
reference sources present (as on a machine that only receives the built
files) it does nothing and returns.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("MLBM_REFERENCE_DIR", "/root/reference")

# 16x12x10 / 24x20x18: small non-cubic parity boxes; 40^3: positions file at
# resolution 0.2; 64^3: periodic phase-separation case; 200^3: drainage case.
SIZES = ["16x12x10", "24x20x18", "40x40x40", "64x64x64", "200x200x200"]

CXXFLAGS = ["-O2", "-std=c++14", "-fopenmp", "-fPIC", "-ffp-contract=off",
            "-w"]


def _prepare_tree(size: str, scratch: str) -> str:
    lx, ly, lz = (int(v) for v in size.split("x"))
    root = os.path.join(scratch, f"ref_{size}")
    if os.path.isdir(root):
        shutil.rmtree(root)
    for sub in ("include", "src", "external"):
        shutil.copytree(os.path.join(REFERENCE, sub), os.path.join(root, sub))
    model = os.path.join(root, "include", "lbm_model.cuh")
    os.chmod(model, 0o644)
    text = open(model).read()
    for name, val in (("lx", lx), ("ly", ly), ("lz", lz)):
        text, n = re.subn(rf"#define {name} \d+", f"#define {name} {val}", text)
        if n != 1:
            raise RuntimeError(f"could not set {name} in {model}")
    with open(model, "w") as fh:
        fh.write(text)
    return root


def build(sizes=None, force: bool = False, quiet: bool = True) -> list[str]:
    """Compile the oracle binaries; returns the list of built library paths."""
    if not os.path.isdir(os.path.join(REFERENCE, "include")):
        return []
    sizes = sizes or SIZES
    os.makedirs(OUT, exist_ok=True)
    scratch = os.path.join(tempfile.gettempdir(), "mlbm_ref_build")
    os.makedirs(scratch, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.h")
    harness = os.path.join(HERE, "ref_harness.cpp")
    deps = [shim, harness, os.path.abspath(__file__)]
    built = []
    for size in sizes:
        lib = os.path.join(OUT, f"libref_{size}.so")
        exe = os.path.join(OUT, f"multiphaselbm_cpu_{size}")
        newest_dep = max(os.path.getmtime(d) for d in deps)
        if (not force and os.path.exists(lib) and os.path.exists(exe)
                and os.path.getmtime(lib) > newest_dep):
            built.append(lib)
            continue
        root = _prepare_tree(size, scratch)
        inc = ["-include", shim, "-I", os.path.join(root, "include"),
               "-I", os.path.join(root, "external")]
        objs = []
        for src, name in ((harness, "harness.o"),
                          (os.path.join(root, "src", "multiphase_lbm.cu"),
                           "driver.o")):
            obj = os.path.join(root, name)
            cmd = ["g++", *CXXFLAGS, *inc, "-x", "c++", "-c", src, "-o", obj]
            subprocess.run(cmd, check=True,
                           stdout=subprocess.DEVNULL if quiet else None)
            objs.append(obj)
        subprocess.run(["g++", "-shared", "-fopenmp", *objs, "-o", lib],
                       check=True)
        main_o = os.path.join(root, "main.o")
        subprocess.run(["g++", *CXXFLAGS, *inc, "-x", "c++", "-c",
                        os.path.join(root, "src", "main.cc"), "-o", main_o],
                       check=True)
        subprocess.run(["g++", "-fopenmp", main_o, *objs, "-o", exe],
                       check=True)
        built.append(lib)
        if not quiet:
            print("built", lib)
    return built


# The reference's own host driver (src/multiphase_lbm.cu, src/main.cc)
# linked against libmlbm through include/mlbm_compat.h instead of its CUDA
# kernels: the drop-in demonstration.  Its iteration_host.h is replaced by a
# generated three-line header that includes mlbm_compat.h.
COMPAT_HEADER = """#ifndef ITERATION_HOST_H_
#define ITERATION_HOST_H_
#include <cuda_runtime.h>
#include "lbm_model.cuh"
#include "mlbm_compat.h"
#define cudaErrorCheck(ans) { mlbm_compat_check((int)(ans), __FILE__, __LINE__); }
#endif
"""


def build_dropin(sizes=None, force: bool = False) -> list[str]:
    """Build oracle/_ref/refdriver_b200_<size>: the reference driver running
    the B200 kernels (needs libmlbm.so built first)."""
    if not os.path.isdir(os.path.join(REFERENCE, "include")):
        return []
    root_repo = os.path.dirname(HERE)
    lib = os.path.join(root_repo, "multiphase_lbm_b200", "libmlbm.so")
    if not os.path.exists(lib):
        return []
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    scratch = os.path.join(tempfile.gettempdir(), "mlbm_ref_build")
    out = []
    for size in sizes or SIZES:
        exe = os.path.join(OUT, f"refdriver_b200_{size}")
        if (not force and os.path.exists(exe)
                and os.path.getmtime(exe) > os.path.getmtime(lib)):
            out.append(exe)
            continue
        root = _prepare_tree(size, scratch)
        gen = os.path.join(root, "compat_include")
        os.makedirs(gen, exist_ok=True)
        with open(os.path.join(gen, "iteration_host.h"), "w") as fh:
            fh.write(COMPAT_HEADER)
        cmd = [nvcc, "-O2", "-std=c++14", "-w", "-Xcompiler", "-fopenmp",
               "-gencode", "arch=compute_100a,code=sm_100a",
               "-I", gen, "-I", os.path.join(root, "include"),
               "-I", os.path.join(root, "external"),
               "-I", os.path.join(root_repo, "include"),
               os.path.join(root, "src", "multiphase_lbm.cu"),
               os.path.join(root, "src", "main.cc"),
               "-L", os.path.dirname(lib), "-lmlbm",
               "-Xlinker", "-rpath,$ORIGIN/../../multiphase_lbm_b200",
               "-o", exe]
        subprocess.run(cmd, check=True)
        out.append(exe)
    return out


# The reference's own CUDA time step (src/iteration_host.cu, unmodified)
# with its host driver (src/multiphase_lbm.cu) for the set-up, driven by
# oracle/ref_cuda_timer.cu, which times multiphaselbm_iteration between CUDA
# events: the reference's CUDA path measured on the B200 beside this library.
# Not a parity oracle (its collision kernel reads neighbours another thread
# may be writing, so its results are not deterministic).
CUDA_SIZES = ["64x64x64", "200x200x200"]


def cuda_timer_path(size: str = "200x200x200") -> str:
    return os.path.join(OUT, f"ref_cuda_timer_{size}")


def build_cuda(sizes=None, force: bool = False) -> list[str]:
    """Build oracle/_ref/ref_cuda_timer_<size>."""
    if not os.path.isdir(os.path.join(REFERENCE, "include")):
        return []
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    scratch = os.path.join(tempfile.gettempdir(), "mlbm_ref_build")
    os.makedirs(OUT, exist_ok=True)
    timer = os.path.join(HERE, "ref_cuda_timer.cu")
    out = []
    for size in sizes or CUDA_SIZES:
        exe = cuda_timer_path(size)
        if (not force and os.path.exists(exe)
                and os.path.getmtime(exe) > os.path.getmtime(timer)):
            out.append(exe)
            continue
        root = _prepare_tree(size, scratch)
        cmd = [nvcc, "-O3", "-std=c++14", "-w", "-Xcompiler", "-fopenmp",
               "-gencode", "arch=compute_100a,code=sm_100a",
               "-I", os.path.join(root, "include"),
               "-I", os.path.join(root, "external"),
               timer, os.path.join(root, "src", "iteration_host.cu"),
               os.path.join(root, "src", "multiphase_lbm.cu"), "-o", exe]
        subprocess.run(cmd, check=True)
        out.append(exe)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--sizes", default=",".join(SIZES))
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    libs = build(args.sizes.split(","), force=args.force, quiet=False)
    libs += build_dropin(args.sizes.split(","), force=args.force)
    libs += build_cuda(force=args.force)
    if not libs:
        print("reference sources not present; nothing built")
    return 0


if __name__ == "__main__":
    sys.exit(main())
