"""GPU cluster statistics (mlbm_cluster_stats_gpu) against the host
calc_cluster restatement (mlbm_cluster_stats, itself pinned to the
reference's host code in test_host_driver.py): cluster counts, the liquid and
gas cluster numbers of every node, cluster order, wet coordination number,
single-cluster radius and boundary ratios, all bit for bit."""
import numpy as np
import pytest

import oracle
from multiphase_lbm_b200 import driver, host

pytestmark = pytest.mark.gpu

RHOL, RHOG = 0.2726, 0.0484
FIELDS = ("liq_cluster_count", "gas_cluster_count", "cluster_order",
          "wet_coord_num", "cluster_radius", "liquid_solid_boundary",
          "liquid_vapor_boundary")


def _same(a, b):
    return (np.isnan(a) and np.isnan(b)) or a == b


def _check(rho, fl, sn, solid_count):
    want, wl, wg = driver.cluster_stats(rho, fl, sn, RHOL, RHOG, solid_count)
    got, gl, gg = driver.cluster_stats(rho, fl, sn, RHOL, RHOG, solid_count,
                                       device=0)
    for k in FIELDS:
        assert _same(got[k], want[k]), (k, got[k], want[k])
    assert np.array_equal(gl, wl)
    assert np.array_equal(gg, wg)
    return got


def _packed(shape, seed, rmin=2.0, rmax=3.5, density=0.7):
    _, sp = host.generate_packing(shape, rmin, rmax, density, seed=seed)
    sn = np.zeros(shape, np.int64)
    fl = np.ones(shape, np.uint8)
    for k, (x, y, z, r) in enumerate(sp):
        host.place_sphere(fl, x, y, z, r, sn, k + 1)
    return fl, sn, len(sp)


def _smooth(shape, seed, passes=3):
    f = np.random.default_rng(seed).normal(size=shape)
    for _ in range(passes):
        f = (f + np.roll(f, 1, 0) + np.roll(f, -1, 0) + np.roll(f, 1, 1)
             + np.roll(f, -1, 1) + np.roll(f, 1, 2) + np.roll(f, -1, 2)) / 7
    return f


@pytest.mark.parametrize("shape,seed", [((24, 20, 18), 1), ((24, 20, 18), 2),
                                        ((64, 48, 40), 3), ((3, 17, 5), 4),
                                        ((1, 9, 11), 5)])
def test_random_fields_match_host(shape, seed):
    if min(shape) >= 8:
        fl, sn, ns = _packed(shape, seed)
    else:
        rng = np.random.default_rng(seed)
        fl = (rng.random(shape) > 0.2).astype(np.uint8)
        sn = np.where(fl == 0, rng.integers(1, 6, size=shape), 0).astype(np.int64)
        ns = 5
    rho = (0.15 + 1.5 * _smooth(shape, seed)).astype(np.float32)
    got = _check(rho, fl, sn, ns)
    assert got["liq_cluster_count"] > 0 or min(shape) < 8


def test_matches_reference_build_when_present():
    """Against the reference's own calc_cluster compiled for the CPU."""
    shape = (24, 20, 18)
    if tuple(shape) not in oracle.reference_sizes():
        pytest.skip(f"oracle/_ref has no {shape} build")
    ref = oracle.Reference(shape)
    fl, sn, ns = _packed(shape, 7)
    rho = (0.15 + 1.5 * _smooth(shape, 7)).astype(np.float32)
    want, wl, wg = ref.driver_clusters(rho, rho.copy(), fl, sn, ns, RHOL, RHOG)
    got, gl, gg = driver.cluster_stats(rho, fl, sn, RHOL, RHOG, ns, device=0)
    assert got["liq_cluster_count"] == want["liq_cluster_count"]
    assert got["gas_cluster_count"] == want["gas_cluster_count"]
    assert np.array_equal(gl, wl) and np.array_equal(gg, wg)
    for k in ("cluster_order", "wet_coord_num", "cluster_radius",
              "liquid_solid_boundary", "liquid_vapor_boundary"):
        a, b = got[k], want[k]
        assert (np.isnan(a) and np.isnan(b)) or a == pytest.approx(b, rel=1e-6), k


@pytest.mark.parametrize("wrap", ["x", "y", "z", "xyz", "none"])
def test_single_cluster_radius_with_periodic_wrap(wrap):
    shape = (24, 20, 18)
    fl = np.ones(shape, np.uint8)
    sn = np.zeros(shape, np.int64)
    x, y, z = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    c = [11, 10, 9]
    for ax, name in enumerate("xyz"):
        if name in wrap:
            c[ax] = 1

    def pd(a, c0, n):
        return np.minimum(np.abs(a - c0), n - np.abs(a - c0))
    d2 = pd(x, c[0], shape[0]) ** 2 + pd(y, c[1], shape[1]) ** 2 \
        + pd(z, c[2], shape[2]) ** 2
    rho = np.where(d2 < 30, 1.5, 0.03).astype(np.float32)
    got = _check(rho, fl, sn, 0)
    assert got["liq_cluster_count"] == 1
    assert got["cluster_radius"] > 0


def test_no_solid_contact_gives_nan_order():
    shape = (20, 20, 20)
    fl = np.ones(shape, np.uint8)
    sn = np.zeros(shape, np.int64)
    rho = np.full(shape, 0.03, np.float32)
    rho[2:6, 2:6, 2:6] = 1.5
    rho[10:14, 10:14, 10:14] = 1.5
    got = _check(rho, fl, sn, 0)
    assert got["liq_cluster_count"] == 2 and np.isnan(got["cluster_order"])


def test_small_clusters_dropped_and_empty_classes():
    shape = (16, 16, 16)
    fl = np.ones(shape, np.uint8)
    sn = np.zeros(shape, np.int64)
    rho = np.full(shape, 0.1, np.float32)  # neither liquid nor gas
    got = _check(rho, fl, sn, 0)
    assert got["liq_cluster_count"] == 0 and got["gas_cluster_count"] == 0
    rho[1:3, 1:3, 1] = 1.5  # 4 nodes: dropped
    rho[8:10, 8:10, 8:10] = 1.5  # 8 nodes: kept
    rho[0, 0, 0:6] = 0.01  # 6 gas nodes: dropped
    rho[5, 5, 0:7] = 0.01  # 7 gas nodes: kept
    got = _check(rho, fl, sn, 0)
    assert got["liq_cluster_count"] == 1 and got["gas_cluster_count"] == 1


def test_drainage_sized_lattice_matches_host():
    """A 160^3 sphere packing with a mixed liquid / gas field."""
    shape = (160, 160, 160)
    fl, sn, ns = _packed(shape, 11, 6.0, 12.0, 0.6)
    rho = (0.15 + 6.0 * _smooth(shape, 11, 4)).astype(np.float32)
    got = _check(rho, fl, sn, ns)
    assert got["liq_cluster_count"] > 1 and got["gas_cluster_count"] > 1


def test_simulated_drainage_field_matches_host():
    """Clusters of a density field the lattice itself produced (64^3
    packing, 300 drainage steps), not only synthetic fields."""
    from conftest import sphere_case

    from multiphase_lbm_b200 import capi
    shape = (64, 64, 64)
    fluid, rho0 = sphere_case(shape, seed=21, rmin=3.0, rmax=7.0,
                              porosity=0.55, rho0=1.9, amp=0.05)
    lat = capi.Lattice(shape)
    lat.set_params(capi.default_params(G=-5.0, rhos=0.223144, tau=1.0,
                                       inlet_width=4, outlet_width=1,
                                       rho_inlet=0.10, rho_outlet=1.95))
    lat.upload(fluid, rho0)
    lat.initialize()
    lat.iterate(0, 300)
    rho = lat.field("rho")
    lat.close()
    sn = np.where(fluid == 0, 1 + (np.arange(fluid.size).reshape(shape) % 9),
                  0).astype(np.int64)
    got = _check(rho, fluid, sn, 9)
    assert got["liq_cluster_count"] >= 1
