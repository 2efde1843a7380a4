"""Slab decomposition on one GPU (slab.py, mlbm_set_slab / mlbm_step_pass /
mlbm_halo_segments): the lattice split along z into 2-4 slabs that exchange
their halos between the passes must reproduce the undecomposed lattice bit
for bit -- populations, density and velocity -- through both AA phases, for
FP32 and FP16 storage, even and uneven splits, one-plane slabs, drainage
slabs and injection.  The slabs run one after another on one stream with
the transport: the ring kernel (one launch per exchange) or torch copies; no
kernel waits on another."""
import numpy as np
import pytest

from conftest import sphere_case

pytestmark = pytest.mark.gpu

DRAIN = dict(G=-5.0, rhos=0.223144, tau=1.0, inlet_width=3, outlet_width=1,
             rho_inlet=0.17, rho_outlet=1.90)


def _whole(capi, fluid, rho, storage, params):
    lat = capi.Lattice(fluid.shape, storage=storage)
    lat.set_step_kernel(capi.KERNEL_COMPACT)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    return lat


def _compare(shape, parts, storage, steps, params_kw, seed=5, transport="ring"):
    import torch

    from multiphase_lbm_b200 import capi, slab
    fluid, rho = sphere_case(shape, seed=seed, rmin=2.5, rmax=5.0,
                             porosity=0.55, rho0=1.9, amp=0.05)
    params = capi.default_params(**params_kw)
    whole = _whole(capi, fluid, rho, storage, params)
    run = slab.decompose(fluid, rho, params, parts, storage,
                         transport=transport)
    try:
        whole.iterate(0, steps, write_velocity=True)
        run.run(0, steps - 1)
        run.step(steps - 1, write_velocity=True)
        torch.cuda.synchronize()
        m = fluid.astype(bool)
        for which in ("f", "rho", "velocity"):
            a = whole.field(which)
            b = slab.gather(run.slabs, which)
            assert np.array_equal(a[m], b[m]), (which, shape, parts, steps)
    finally:
        run.close()
        whole.close()


@pytest.mark.parametrize("transport", ["ring", "local"])
@pytest.mark.parametrize("parts", [2, 3, 4])
@pytest.mark.parametrize("steps", [1, 2, 7])
def test_slabs_match_whole_lattice_fp32(parts, steps, transport):
    from multiphase_lbm_b200 import capi
    _compare((40, 36, 32), parts, capi.STORE_F32, steps, DRAIN,
             transport=transport)


@pytest.mark.parametrize("transport", ["ring", "local"])
@pytest.mark.parametrize("parts", [2, 3])
def test_slabs_match_whole_lattice_fp16(parts, transport):
    from multiphase_lbm_b200 import capi
    _compare((40, 36, 32), parts, capi.STORE_F16, 8, DRAIN, transport=transport)


def test_one_plane_slabs_and_odd_rows():
    # 6 slabs over 6 planes: every slab has one own plane, whose edge on both
    # faces is the same plane
    _compare((37, 20, 6), 6, 0, 5, DRAIN, seed=9)


def test_single_slab_is_its_own_neighbour():
    _compare((32, 24, 20), 1, 0, 6, DRAIN)


def test_injection_steps_match():
    kw = dict(DRAIN, rho_inject_period=2, rho_increment=0.01)
    _compare((40, 36, 32), 3, 0, 6, kw, seed=13)


def test_slab_refuses_whole_lattice_calls():
    from multiphase_lbm_b200 import capi, slab
    fluid, rho = sphere_case((32, 24, 20), seed=1, rmin=2.5, rmax=5.0,
                             porosity=0.55, rho0=1.9, amp=0.05)
    run = slab.decompose(fluid, rho, capi.default_params(**DRAIN), 2)
    try:
        lat = run.slabs[0].lat
        with pytest.raises(capi.MlbmError, match="mlbm_step_pass"):
            lat.iterate(0, 1)
        with pytest.raises(capi.MlbmError, match="halo planes"):
            lat.stats()
        with pytest.raises(capi.MlbmError):
            lat.step_pass(0, 2)
    finally:
        run.close()


@pytest.mark.parametrize("storage_name,steps", [("STORE_F32", 101), ("STORE_F16", 50)])
def test_long_run_four_slabs(storage_name, steps):
    """Many steps through both AA phases: the decomposition stays bit for bit
    on the whole lattice's trajectory (drainage boundary, 64^3)."""
    from multiphase_lbm_b200 import capi
    _compare((64, 64, 64), 4, getattr(capi, storage_name), steps, DRAIN,
             seed=17)


def test_ring_refuses_slabs_of_different_lattices():
    """A ring whose neighbouring halo and edge planes differ in size is
    refused at creation (the kernel would copy past a plane)."""
    from multiphase_lbm_b200 import capi, slab
    fa, ra = sphere_case((32, 24, 20), seed=1, rmin=2.5, rmax=5.0,
                         porosity=0.55, rho0=1.9, amp=0.05)
    fb, rb = sphere_case((32, 24, 20), seed=2, rmin=2.5, rmax=5.0,
                         porosity=0.55, rho0=1.9, amp=0.05)
    p = capi.default_params(**DRAIN)
    a = slab.Slab(fa, ra, p, 0, 10)
    b = slab.Slab(fb, rb, p, 10, 10)
    try:
        with pytest.raises(capi.MlbmError, match="halo and edge"):
            slab.RingExchange([a, b])
        whole = _whole(capi, fa, ra, capi.STORE_F32, p)
        with pytest.raises(capi.MlbmError, match="not a slab"):
            whole.halo_segments(capi.HALO_POP_EDGE, 0)
        whole.close()
    finally:
        a.close()
        b.close()
