"""The one-pass step (KERNEL_BAND): one launch per step that reads the step's
populations from one buffer and pushes the new ones into a second buffer,
with psi of each band of rows formed in shared memory plane by plane.  Same
loads and the same arithmetic per node as the two-pass kernels, so the
results must be bit-identical to them for every band shape, including bands
that wrap onto themselves (fewer rows than a band plus its two halo rows),
single planes and one-node rows.  Against the oracle (the reference's
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


def _lattice(capi, shape, fluid, rho, kernel, storage=0, band=None, **kw):
    lat = capi.Lattice(shape, storage=storage)
    lat.set_step_kernel(kernel)
    if band:
        lat.set_band_shape(*band)
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


def test_band_limits():
    from multiphase_lbm_b200 import capi
    lat = capi.Lattice((16, 16, 16), storage=capi.STORE_F16)
    lat.set_step_kernel(capi.KERNEL_BAND)
    assert lat.step_kernel == capi.KERNEL_BAND
    with pytest.raises(capi.MlbmError):
        capi.Lattice((16, 16, 16), storage=capi.STORE_F64).set_step_kernel(
            capi.KERNEL_BAND)
    with pytest.raises(capi.MlbmError):
        lat.set_band_shape(0, 4)
    with pytest.raises(capi.MlbmError):
        lat.set_band_shape(4, 0)



def test_band_rows_too_long_for_shared_memory_run_as_compact():
    """Rows of 2000 nodes: not even a band of one row (three staged rows)
    fits shared memory, so BAND steps run as COMPACT steps -- the same bits."""
    from multiphase_lbm_b200 import capi
    shape = (2000, 4, 3)
    fluid, rho = sphere_case(shape, seed=1, rmin=1.0, rmax=1.5, porosity=0.7,
                             rho0=1.5, amp=0.2)
    a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN), 6)
    b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **DRAIN), 6)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_band_matches_oracle_drainage_100_steps():
    from multiphase_lbm_b200 import capi
    shape = (64, 48, 40)
    fluid, rho = sphere_case(shape, seed=11, rmin=3.0, rmax=6.0, porosity=0.55,
                             rho0=1.9, amp=0.02)
    lat = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
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


# odd shapes: one-node rows, single plane, two planes, three rows (every band
# wraps onto itself), rows shorter than a mask word, rows of several words
SHAPES = [(40, 32, 24), (33, 5, 7), (70, 3, 2), (300, 6, 6), (1, 9, 8),
          (24, 20, 1), (17, 2, 9)]


@pytest.mark.parametrize("storage", [0, 1])
@pytest.mark.parametrize("shape", SHAPES)
def test_band_bit_identical_to_two_pass(shape, storage):
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(shape, seed=sum(shape) + storage, rmin=1.5,
                             rmax=3.5, porosity=0.6, rho0=1.5, amp=0.3)
    kw = dict(G=-5.0, rhos=0.223144, tau=1.0, rho_shift=1.0)
    if shape[0] >= 8:
        kw.update(inlet_width=2, outlet_width=1, rho_inlet=0.17, rho_outlet=1.9)
    b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS,
                      storage=storage, **kw))
    for band in [(1, 1), (2, 3), (4, 24), (64, 1000)]:
        a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_BAND,
                          storage=storage, band=band, **kw))
        for u, v in zip(a, b):
            assert np.array_equal(u, v), band


def test_band_with_injection_bit_identical():
    """The injection band (y < inject_position * ly on steps that are
    multiples of the period) and reverse/inject-type arguments."""
    from multiphase_lbm_b200 import capi
    shape = (48, 40, 32)
    fluid, rho = sphere_case(shape, seed=3, rmin=2.0, rmax=5.0, porosity=0.55,
                             rho0=0.7, amp=0.05)
    kw = dict(G=-5.0, rhos=0.223144, tau=1.0, rho_inject_period=3,
              rho_increment=0.002, inject_position=0.25)
    outs = []
    for kind in (capi.KERNEL_BAND, capi.KERNEL_TWO_PASS):
        lat = _lattice(capi, shape, fluid, rho, kind, **kw)
        for s0, rev, typ in ((0, 1, 0), (7, -1, 1), (14, 1, 2)):
            lat.iterate(s0, 7, reverse=rev, inject_type=typ)
        outs.append((lat.field("rho"), lat.field("f")))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_band_large_lattice_many_blocks():
    """Thousands of blocks per step, neighbouring bands in flight at once:
    bit-identical to the compact two-pass step over 40 steps, FP32 and FP16."""
    from multiphase_lbm_b200 import capi
    shape = (160, 144, 128)
    fluid, rho = sphere_case(shape, seed=7, rmin=4.0, rmax=10.0, porosity=0.5,
                             rho0=2.0, amp=0.01)
    kw = dict(DRAIN, rho_shift=1.0)
    for storage in (0, 1):
        a = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_BAND,
                          storage=storage, band=(3, 16), **kw), 40)
        b = _run(_lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT,
                          storage=storage, **kw), 40)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


def test_band_switching():
    """band -> two-pass -> compact -> band -> two-pass -> band against
    two-pass throughout, with odd step counts so each switch meets the other
    AA phase."""
    from multiphase_lbm_b200 import capi
    shape = (64, 40, 36)
    fluid, rho = sphere_case(shape, seed=2, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=1.9, amp=0.02)
    a = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
    b = _lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **DRAIN)
    step = 0
    for kind, n in ((capi.KERNEL_BAND, 11), (capi.KERNEL_TWO_PASS, 5),
                    (capi.KERNEL_COMPACT, 3), (capi.KERNEL_BAND, 6),
                    (capi.KERNEL_TWO_PASS, 7), (capi.KERNEL_BAND, 4)):
        a.set_step_kernel(kind)
        a.iterate(step, n)
        b.iterate(step, n)
        step += n
    assert np.array_equal(a.field("rho"), b.field("rho"))
    assert np.array_equal(a.field("f"), b.field("f"))


def test_band_wait_limit_runs_out_and_the_context_recovers():
    """A hand-over wait that nothing completes (mlbm_test_stall_wait) ends
    after the wait limit with MLBM_ERR_TIMEOUT instead of hanging; the
    device stays usable and the lattice, initialised again, gives what a
    fresh lattice gives."""
    from multiphase_lbm_b200 import capi
    shape = (48, 40, 36)
    fluid, rho = sphere_case(shape, seed=4, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=1.9, amp=0.02)
    lat = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
    lat.set_wait_limit(2_000_000)  # 2 ms
    lat.iterate(0, 3)  # from AA phase 0 the first step is a two-pass step
    lat.synchronize()
    lat.test_stall_wait()
    lat.iterate(3, 1)
    with pytest.raises(capi.MlbmError) as exc:
        lat.synchronize()
    assert exc.value.status == 5  # MLBM_ERR_TIMEOUT
    lat.set_wait_limit(0)
    lat.initialize()
    lat.iterate(0, 9)
    ref = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
    ref.iterate(0, 9)
    assert np.array_equal(lat.field("rho"), ref.field("rho"))
    assert np.array_equal(lat.field("f"), ref.field("f"))
    with pytest.raises(capi.MlbmError):
        _lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT,
                 **DRAIN).test_stall_wait()
