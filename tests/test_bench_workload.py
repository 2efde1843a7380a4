"""The benchmark's 200^3 drainage workload, pinned on the CPU.

* The committed positions file voxelises to the same mask through the
  reference's own command-file parser and read_positions (oracle/_ref) as
  through this library's mlbm_read_positions, and to the mask of the seeded
  generator that wrote it; the reference's initial density is 2.0 at every
  node.
* The oracle (oracle/mlbm_oracle.c) reproduces the reference's own kernels
  (compiled for the CPU, oracle/_ref) bit for bit on that workload, drainage
  slabs included, over the first steps of both AA phases -- so the GPU
  parity tests at this size, which compare against the oracle, compare
  against the reference.
"""
import os
import sys

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402

SHAPE = (200, 200, 200)


def _ref():
    if SHAPE not in oracle.reference_sizes():
        pytest.skip("oracle/_ref has no 200^3 build")
    return oracle.Reference(SHAPE)


def test_positions_file_same_mask_through_both_readers(tmp_path):
    from multiphase_lbm_b200 import host
    ref = _ref()
    r_rho, r_fl, _, info = ref.driver_read(bench.command_file(str(tmp_path)))
    fluid, rho, n = bench.workload()
    assert n == int(info["solid_count"]) == 1075
    assert np.array_equal(r_fl, fluid)
    assert np.all(r_rho == np.float32(2.0)) and np.array_equal(r_rho, rho)
    gen, spheres = host.generate_packing(SHAPE, 5.0, 15.0, 0.50, 2024)
    assert len(spheres) == n and np.array_equal(gen, fluid)
    assert int(fluid.sum()) == 3998416


def test_oracle_bit_exact_with_reference_at_bench_size(tmp_path):
    ref = _ref()
    rho, fluid, _, _ = ref.driver_read(bench.command_file(str(tmp_path)))
    p = oracle.make_params(**bench.PHYS)
    ref.setup(rho, fluid, p)
    port = oracle.Port(rho, fluid, p)
    step = 0
    for n in (1, 2):
        ref.step(step, n)
        port.step(step, n)
        step += n
        for field in ("rho", "f"):
            a, b = ref.get(field), port.get(field)
            assert np.array_equal(a, b), f"step {step}: {field}"
