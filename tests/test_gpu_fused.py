"""The fused persistent time step against the two-pass kernels.

Both run the same per-node arithmetic on the same loads, so after any number
of steps their populations and densities must be bit-identical.  Covers the
schedule's corner cases: one, two and three planes in z, rows blocks that
do not divide ly, row segments (lx > 512), every storage format, drainage,
injection, and custom tuning (rows per item, plane lag).
"""
import numpy as np
import pytest

from conftest import random_case

pytestmark = pytest.mark.gpu

SC = dict(G=-6.0, rhos=0.182322, tau=1.0)


def _run(shape, fluid, rho, kind, storage=0, steps=23, tuning=None, **kw):
    from multiphase_lbm_b200 import capi
    lat = capi.Lattice(shape, storage=storage)
    lat.set_params(capi.default_params(**kw))
    lat.upload(fluid, rho)
    lat.initialize()
    lat.set_step_kernel(kind)
    if tuning:
        lat.set_tuning(*tuning)
    lat.iterate(0, steps - 1)
    lat.iterate(steps - 1, 1, write_velocity=True)
    lat.synchronize()
    out = (lat.field("rho", f64=storage == 2), lat.field("f", f64=storage == 2),
           lat.field("velocity"))
    lat.close()
    return out


@pytest.mark.parametrize("shape", [(32, 16, 1), (40, 12, 2), (24, 9, 3),
                                   (200, 30, 20), (600, 5, 6), (33, 70, 11)])
def test_fused_bit_identical_to_two_pass(shape):
    from multiphase_lbm_b200 import capi
    fluid, rho = random_case(shape, seed=sum(shape))
    a = _run(shape, fluid, rho, capi.KERNEL_FUSED, **SC)
    b = _run(shape, fluid, rho, capi.KERNEL_TWO_PASS, **SC)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("storage", [0, 1, 2])
def test_fused_storage_formats(storage):
    from multiphase_lbm_b200 import capi
    shape = (48, 20, 16)
    fluid, rho = random_case(shape, seed=3, rho0=1.0, amp=0.05)
    kw = dict(SC, inlet_width=2, outlet_width=1, rho_inlet=0.1,
              rho_outlet=1.9, rho_increment=0.003, rho_inject_period=4,
              inject_density=1, inject_position=0.5)
    a = _run(shape, fluid, rho, capi.KERNEL_FUSED, storage=storage, **kw)
    b = _run(shape, fluid, rho, capi.KERNEL_TWO_PASS, storage=storage, **kw)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("tuning", [(1, 2), (2, 3), (4, 7), (16, 50)])
def test_fused_tuning_variants(tuning):
    from multiphase_lbm_b200 import capi
    shape = (64, 21, 13)
    fluid, rho = random_case(shape, seed=5)
    a = _run(shape, fluid, rho, capi.KERNEL_FUSED, tuning=tuning, **SC)
    b = _run(shape, fluid, rho, capi.KERNEL_TWO_PASS, **SC)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
