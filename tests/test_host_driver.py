"""The host driver against the reference's own host driver (oracle/_ref):
command-file parsing, geometry and initial density bit for bit, and the
cluster statistics of calc_cluster."""
import os

import numpy as np
import pytest

import oracle
from multiphase_lbm_b200 import driver, host

REF = (40, 40, 40)


def _need_ref(shape):
    if tuple(shape) not in oracle.reference_sizes():
        pytest.skip(f"oracle/_ref has no {shape} build")
    return oracle.Reference(shape)


def _command_file(tmp_path, shape, extra=""):
    _, spheres = host.generate_packing(shape, 2.5, 6.0, 0.6, seed=17)
    pos = str(tmp_path / "grains.txt")
    host.write_positions(pos, spheres)
    text = f"""! command file in the reference's format
result_folder {tmp_path}/RES   ! comment after a value
statPeriod 5
lx {shape[0]}
ly {shape[1]}
lz {shape[2]}
rho0  0.35
IniPerturbRate 0.5
rhos  0.3
G -6.0
tau 1.
rhol_spinodal 0.2725
rhog_spinodal 0.0484
resize
# a hash comment line
resolution 1
read_positions {pos}
place_sphere 10.5 12.25 8.0 3.75
generate_solids 2 2.0 3.0 0 {shape[0]} 0 {shape[1]} 0 {shape[2]}
rho_inject_period 50
rho_increment 0.001
inject_type 1
inject_position 0.5
bogus_token
step_max 30
{extra}
"""
    path = tmp_path / "input.txt"
    path.write_text(text)
    return str(path)


def test_command_file_geometry_and_density_match_reference(tmp_path):
    ref = _need_ref(REF)
    cmd = _command_file(tmp_path, REF)
    r_rho, r_fl, r_sn, r_info = ref.driver_read(cmd)
    d = driver.Driver()
    d.read(cmd)
    rho, fl, sn = d.arrays()
    assert np.array_equal(fl, r_fl)
    assert np.array_equal(sn, r_sn)
    assert np.array_equal(rho, r_rho)
    info = d.info()
    assert info["solid_count"] == int(r_info["solid_count"])
    assert info["step_max"] == int(r_info["step_max"])
    assert info["statPeriod"] == int(r_info["statPeriod"])
    assert abs(info["packing_density"] - r_info["packing_density"]) < 1e-6
    p = d.params()
    assert p.tau == pytest.approx(r_info["tau"]) and p.G == pytest.approx(r_info["G"])
    assert p.rhos == pytest.approx(r_info["rhos"])
    assert p.inject_density == 1 and p.rho_inject_period == 50
    d.close()


def test_last_token_without_trailing_whitespace_is_ignored(tmp_path):
    """Reference parser semantics: a token at end of file not followed by
    whitespace is never acted on (src/multiphase_lbm.cu:631-725)."""
    ref = _need_ref(REF)
    path = tmp_path / "in.txt"
    path.write_text("lx 40 ly 40 lz 40 resize step_max 77")
    _, _, _, r_info = ref.driver_read(str(path))
    d = driver.Driver()
    d.read(str(path))
    assert d.info()["step_max"] == int(r_info["step_max"])


def test_parser_errors(tmp_path):
    from multiphase_lbm_b200.capi import MlbmError
    d = driver.Driver()
    with pytest.raises(MlbmError) as e:
        d.read(str(tmp_path / "missing.txt"))
    assert e.value.status == 6
    bad = tmp_path / "bad.txt"
    bad.write_text("lx 8 ly 8 lz 8 resize tau abc \n")
    with pytest.raises(MlbmError) as e:
        d.read(str(bad))
    assert e.value.status == 7


def test_g_ads_maps_to_solid_density(tmp_path):
    path = tmp_path / "in.txt"
    path.write_text("G -6.0 G_ads -1.0\nlx 8 ly 8 lz 8 resize \n")
    d = driver.Driver()
    d.read(str(path))
    assert d.params().rhos == pytest.approx(0.182322, abs=1e-6)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cluster_statistics_match_reference(seed):
    shape = (24, 20, 18)
    ref = _need_ref(shape)
    rng = np.random.default_rng(seed)
    fl, sp = host.generate_packing(shape, 2.0, 3.5, 0.7, seed=seed)
    sn = np.zeros(shape, np.int64)
    fl2 = np.ones(shape, np.uint8)
    for k, (x, y, z, r) in enumerate(sp):
        host.place_sphere(fl2, x, y, z, r, sn, k + 1)
    # blobs of liquid and gas: smooth random field
    f = rng.normal(size=shape)
    for _ in range(3):
        f = (f + np.roll(f, 1, 0) + np.roll(f, -1, 0) + np.roll(f, 1, 1)
             + np.roll(f, -1, 1) + np.roll(f, 1, 2) + np.roll(f, -1, 2)) / 7
    rho = (0.15 + 1.5 * f).astype(np.float32)
    pres = rho.copy()
    want, wl, wg = ref.driver_clusters(rho, pres, fl2, sn, len(sp), 0.2726, 0.0484)
    got, gl, gg = driver.cluster_stats(rho, fl2, sn, 0.2726, 0.0484, len(sp))
    assert got["liq_cluster_count"] == want["liq_cluster_count"]
    assert got["gas_cluster_count"] == want["gas_cluster_count"]
    assert np.array_equal(gl, wl) and np.array_equal(gg, wg)
    for k in ("cluster_order", "wet_coord_num", "cluster_radius",
              "liquid_solid_boundary", "liquid_vapor_boundary"):
        a, b = got[k], want[k]
        assert (np.isnan(a) and np.isnan(b)) or a == pytest.approx(b, rel=1e-6), k


def test_single_cluster_radius_matches_reference():
    shape = (24, 20, 18)
    ref = _need_ref(shape)
    fl = np.ones(shape, np.uint8)
    sn = np.zeros(shape, np.int64)
    x, y, z = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    # one liquid blob wrapping across the x boundary
    d2 = (np.minimum(np.abs(x - 1), shape[0] - np.abs(x - 1)) ** 2
          + (y - 10) ** 2 + (z - 9) ** 2)
    rho = np.where(d2 < 30, 1.5, 0.03).astype(np.float32)
    want, wl, _ = ref.driver_clusters(rho, rho, fl, sn, 0, 0.2726, 0.0484)
    got, gl, _ = driver.cluster_stats(rho, fl, sn, 0.2726, 0.0484, 0)
    assert got["liq_cluster_count"] == want["liq_cluster_count"] == 1
    assert got["cluster_radius"] == pytest.approx(want["cluster_radius"], rel=1e-6)
    assert np.array_equal(gl, wl)
