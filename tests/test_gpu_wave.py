"""The wavefront step (KERNEL_WAVE): both passes of the compact two-pass step
in one persistent launch, density tiles a few planes ahead of the update
tiles.  Same loads and the same arithmetic per node as the dense two-pass
kernels, so the results must be bit-identical to them, for every work-item
shape (tile size, lookahead) and at sizes where hundreds of CTAs run tiles of
neighbouring planes concurrently.  Against the oracle (the reference's
algorithm restated on the CPU): the FP32 parity bar, density within 1e-5
relative pointwise and populations within 1e-5 relative to their largest
value over the first 100 steps.
"""
import numpy as np
import pytest

import oracle
from conftest import pointwise_rel_err, rel_err, sphere_case

pytestmark = pytest.mark.gpu

DRAIN = dict(G=-5.0, rhos=0.223144, tau=1.0, inlet_width=3, outlet_width=1,
             rho_inlet=0.17, rho_outlet=1.90)


def _lattice(capi, shape, fluid, rho, kernel, storage=0, wave=None, **kw):
    lat = capi.Lattice(shape, storage=storage)
    lat.set_step_kernel(kernel)
    if wave:
        lat.set_wave_shape(*wave)
    lat.set_params(capi.default_params(**kw))
    lat.upload(fluid, rho)
    lat.initialize()
    return lat


def _run(lat, nsteps=20):
    lat.iterate(0, nsteps)
    lat.iterate(nsteps, 1, write_velocity=True)
    lat.synchronize()
    return (lat.field("rho"), lat.field("f"), lat.field("velocity"),
            lat.field("psi"))


def test_wave_limits():
    from multiphase_lbm_b200 import capi
    lat = capi.Lattice((16, 16, 16), storage=capi.STORE_F16)
    lat.set_step_kernel(capi.KERNEL_WAVE)
    assert lat.step_kernel == capi.KERNEL_WAVE
    with pytest.raises(capi.MlbmError):
        capi.Lattice((16, 16, 16), storage=capi.STORE_F64).set_step_kernel(
            capi.KERNEL_WAVE)
    with pytest.raises(capi.MlbmError):
        lat.set_wave_shape(64, 257)


def test_wave_matches_oracle_drainage_100_steps():
    from multiphase_lbm_b200 import capi
    shape = (64, 48, 40)
    fluid, rho = sphere_case(shape, seed=11, rmin=3.0, rmax=6.0, porosity=0.55,
                             rho0=1.9, amp=0.02)
    lat = _lattice(capi, shape, fluid, rho, capi.KERNEL_WAVE, **DRAIN)
    port = oracle.Port(rho, fluid, oracle.make_params(**DRAIN))
    m = fluid.astype(bool)
    step = 0
    for n in (1, 9, 90):
        lat.iterate(step, n)
        port.step(step, n)
        step += n
        lat.synchronize()
        e = pointwise_rel_err(lat.field("rho"), port.get("rho"), m)
        assert e <= 1e-5, f"step {step}: rho {e:.3e}"
        e = rel_err(lat.field("f"), port.get("f"), m)
        assert e <= 1e-5, f"step {step}: populations {e:.3e}"


# odd shapes: single plane, two planes, rows shorter than a mask word, rows of
# several words, planes whose fluid nodes fill less than one tile
SHAPES = [(40, 32, 24), (33, 5, 7), (70, 3, 2), (300, 6, 6), (1, 9, 8),
          (24, 20, 1)]


@pytest.mark.parametrize("storage", [0, 1])
@pytest.mark.parametrize("shape", SHAPES)
def test_wave_bit_identical_to_two_pass(shape, storage):
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(shape, seed=sum(shape) + storage, rmin=1.5,
                             rmax=3.5, porosity=0.6, rho0=1.5, amp=0.3)
    kw = dict(G=-5.0, rhos=0.223144, tau=1.0, rho_shift=1.0)
    if shape[0] >= 8:
        kw.update(inlet_width=2, outlet_width=1, rho_inlet=0.17, rho_outlet=1.9)
    a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_WAVE,
                      storage=storage, **kw))
    b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS,
                      storage=storage, **kw))
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


# tile nodes x lookahead planes: tiles smaller than a CTA, lookahead 0 (the
# density of plane z+1 right before the update of plane z), lookahead longer
# than the lattice
@pytest.mark.parametrize("wave", [(32, 0), (256, 1), (1000, 3), (4096, 8),
                                  (777, 250)])
def test_wave_shapes_bit_identical(wave):
    from multiphase_lbm_b200 import capi
    shape = (96, 80, 64)
    fluid, rho = sphere_case(shape, seed=21, rmin=2.0, rmax=6.0, porosity=0.5,
                             rho0=1.9, amp=0.05)
    a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_WAVE, wave=wave,
                      **DRAIN), 30)
    b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT, **DRAIN), 30)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_wave_with_injection_bit_identical():
    """The injection band (y < inject_position * ly on steps that are
    multiples of the period) and reverse/inject-type arguments."""
    from multiphase_lbm_b200 import capi
    shape = (48, 40, 32)
    fluid, rho = sphere_case(shape, seed=3, rmin=2.0, rmax=5.0, porosity=0.55,
                             rho0=0.7, amp=0.05)
    kw = dict(G=-5.0, rhos=0.223144, tau=1.0, rho_inject_period=3,
              rho_increment=0.002, inject_position=0.25)
    outs = []
    for kind in (capi.KERNEL_WAVE, capi.KERNEL_TWO_PASS):
        lat = _lattice(capi, shape, fluid, rho, kind, **kw)
        for s0, rev, typ in ((0, 1, 0), (7, -1, 1), (14, 1, 2)):
            lat.iterate(s0, 7, reverse=rev, inject_type=typ)
        outs.append((lat.field("rho"), lat.field("f")))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_wave_large_lattice_many_ctas():
    """A lattice with thousands of work items per step, so that every SM runs
    tiles of several planes at once: bit-identical to the compact two-pass
    step over 40 steps, FP32 and FP16."""
    from multiphase_lbm_b200 import capi
    shape = (160, 144, 128)
    fluid, rho = sphere_case(shape, seed=7, rmin=4.0, rmax=10.0, porosity=0.5,
                             rho0=2.0, amp=0.01)
    kw = dict(DRAIN, rho_shift=1.0)
    for storage in (0, 1):
        a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_WAVE,
                          storage=storage, wave=(512, 4), **kw), 40)
        b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT,
                          storage=storage, **kw), 40)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


def test_wave_switching_and_autotune():
    """wave -> two-pass -> wave (after autotune) -> single-pass -> wave, against
    two-pass throughout; the autotuned shape is one of the candidates."""
    from multiphase_lbm_b200 import capi
    shape = (64, 40, 36)
    fluid, rho = sphere_case(shape, seed=2, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=1.9, amp=0.02)
    a = _lattice(capi, shape, fluid, rho, capi.KERNEL_WAVE, **DRAIN)
    b = _lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **DRAIN)
    step = 0
    a.iterate(step, 11)
    b.iterate(step, 11)
    step += 11
    a.set_step_kernel(capi.KERNEL_TWO_PASS)
    a.iterate(step, 5)
    b.iterate(step, 5)
    step += 5
    a.set_step_kernel(capi.KERNEL_WAVE)
    tile, ahead, done = a.autotune(step, trial_steps=2)
    assert tile in (256, 512, 1024, 2048) and ahead in (1, 2, 4, 8, 16)
    assert done > 0
    b.iterate(step, done)
    step += done
    for kind in (capi.KERNEL_SINGLE_PASS, capi.KERNEL_WAVE):
        a.set_step_kernel(kind)
        a.iterate(step, 7)
        b.iterate(step, 7)
        step += 7
    m = fluid.astype(bool)
    assert pointwise_rel_err(a.field("rho"), b.field("rho"), m) <= 1e-5
    assert rel_err(a.field("f"), b.field("f"), m) <= 1e-5
    with pytest.raises(capi.MlbmError):
        a.set_wave_shape(8, 4)           # fewer than 32 nodes per item
