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
* The 64^3 periodic comparison case reads the same geometry and initial
  density in both arms (the reference's parser on the command file its CUDA
  build is timed with; this library's readers on the same positions file).
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


def test_periodic_64_case_same_geometry_and_density_in_both_arms(tmp_path):
    """The 64^3 periodic comparison case: the command file the reference arm
    gives the reference's CUDA build, read by the reference's own parser,
    yields the mask and initial density (its srand(1)/rand() perturbation)
    that this library's arm builds from the same positions file."""
    from multiphase_lbm_b200 import host
    shape = bench.SHAPE_64
    if shape not in oracle.reference_sizes():
        pytest.skip("oracle/_ref has no 64^3 build")
    ref = oracle.Reference(shape)
    r_rho, r_fl, _, info = ref.driver_read(bench.command_file_64(str(tmp_path)))
    fluid, _, n = host.read_positions(bench.POSITIONS_64, shape)
    rho = host.init_density(shape, 0.70, bench.RATE_64)
    assert n == int(info["solid_count"]) == 276
    assert np.array_equal(r_fl, fluid) and int(fluid.sum()) == 131062
    assert np.array_equal(r_rho[fluid == 1], rho[fluid == 1])
    gen, spheres = host.generate_packing(shape, 2.5, 7.5, 0.50, 64)
    assert len(spheres) == n and np.array_equal(gen, fluid)
