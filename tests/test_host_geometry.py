"""Host geometry of libmlbm against the reference's own host driver.

The golden fixture voxel_40.npz holds the mask, solid numbers and initial
density the reference's read_data produced (oracle/_ref, see
tests/golden/make_golden.py) for: resize with rho0 0.7 / IniPerturbRate
0.0285714, read_positions of a seeded positions file, one place_sphere and
generate_solids 3 ... ; libmlbm must reproduce them bit for bit.
"""
import os

import numpy as np
import pytest

import oracle
from multiphase_lbm_b200 import host

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_voxeliser_density_and_solids_bit_exact(tmp_path):
    d = np.load(os.path.join(GOLDEN, "voxel_40.npz"))
    shape = d["fluid"].shape
    rho = host.init_density(shape, 0.7, 0.0285714)
    assert np.array_equal(rho, d["rho"])
    pos = str(tmp_path / "pos.txt")
    host.write_positions(pos, d["spheres"])
    fluid, sn, count = host.read_positions(pos, shape, 1.0)
    # the reference computes the packing density right after read_positions
    # (src/multiphase_lbm.cu:690-691)
    pd = host.packing_density(fluid)
    # the place_sphere token does not advance the grain counter
    # (src/multiphase_lbm.cu:669-674): its nodes carry the current count
    host.place_sphere(fluid, 3.5, 35.25, 20.0, 4.75, sn, count)
    # generate_solids continues the C library rand() stream after the
    # density initialisation, exactly like the reference's read_data
    host.init_density(shape, 0.7, 0.0285714)
    count = _generate_solids(fluid, sn, 3, 2.0, 4.0, 0, 40, 0, 40, 0, 40,
                             count)
    assert np.array_equal(fluid, d["fluid"])
    assert np.array_equal(sn, d["solid_number"])
    assert count == int(d["solid_count"])
    assert abs(pd - float(d["packing_density"])) < 1e-6


def _generate_solids(fluid, sn, num, rmin, rmax, x0, x1, y0, y1, z0, z1,
                     count):
    import ctypes as C
    n = C.c_int64(count)
    from multiphase_lbm_b200.capi import check
    check(host.hlib().mlbm_generate_solids(
        fluid.ctypes.data, sn.ctypes.data, *fluid.shape, num, rmin, rmax,
        x0, x1, y0, y1, z0, z1, C.byref(n)))
    return n.value


@pytest.mark.parametrize("shape,res", [((64, 64, 64), 1.0),
                                       ((24, 20, 18), 0.5)])
def test_voxeliser_against_reference_live(tmp_path, shape, res):
    if tuple(shape) not in oracle.reference_sizes():
        pytest.skip("no oracle/_ref build of this size")
    _, spheres = host.generate_packing(shape, 2.5, 7.5, 0.55, seed=99)
    spheres = spheres / np.float32(res)  # positions scaled back by resolution
    pos = str(tmp_path / "pos.txt")
    host.write_positions(pos, spheres)
    cmd = tmp_path / "in.txt"
    cmd.write_text(f"resize\nresolution {res}\nread_positions {pos}\n")
    ref = oracle.Reference(shape)
    _, rfl, rsn, info = ref.driver_read(str(cmd))
    fluid, sn, count = host.read_positions(pos, shape, res)
    assert np.array_equal(fluid, rfl)
    assert np.array_equal(sn, rsn)
    assert count == int(info["solid_count"])


def test_example_positions_file_porosity():
    """The reference's example packing at 200^3, resolution 1: porosity
    0.50187 (the reference voxelisation)."""
    from oracle import build_ref
    path = os.path.join(build_ref.REFERENCE, "example_positions_file")
    if not os.path.exists(path):
        pytest.skip("reference example file not present")
    fluid, _, count = host.read_positions(path, (200, 200, 200), 1.0)
    assert count == 767
    assert abs(fluid.mean() - 0.50187) < 5e-6


def test_generate_packing_reaches_target_and_is_seeded():
    a, sa = host.generate_packing((48, 40, 32), 2.5, 7.5, 0.5, seed=3)
    b, sb = host.generate_packing((48, 40, 32), 2.5, 7.5, 0.5, seed=3)
    c, _ = host.generate_packing((48, 40, 32), 2.5, 7.5, 0.5, seed=4)
    assert np.array_equal(a, b) and np.array_equal(sa, sb)
    assert not np.array_equal(a, c)
    assert a.mean() <= 0.5 and a.mean() > 0.45
    # the spheres reproduce the mask through the reference voxeliser rule
    fl = np.ones_like(a)
    for x, y, z, r in sa:
        host.place_sphere(fl, x, y, z, r)
    assert np.array_equal(fl, a)


def test_positions_file_errors(tmp_path):
    from multiphase_lbm_b200.capi import MlbmError
    bad = tmp_path / "bad.txt"
    bad.write_text("1.0\n2.0\nthree\n4.0\n")
    with pytest.raises(MlbmError) as e:
        host.read_positions(str(bad), (8, 8, 8))
    assert e.value.status == 7
    with pytest.raises(MlbmError) as e:
        host.read_positions(str(tmp_path / "missing.txt"), (8, 8, 8))
    assert e.value.status == 6
