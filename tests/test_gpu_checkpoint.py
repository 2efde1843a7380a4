"""Exact checkpoints (mlbm_checkpoint_*): save a lattice at step k, load the
image into a fresh lattice of the same size and storage, run m more steps:
density, populations and velocity are bit-identical to the lattice that ran
k + m steps uninterrupted -- FP32, FP16 and FP64 storage, from either AA
phase (odd and even k), through memory and through a file, with the step
kernels that hold the state in the fluid-only layout.  Images of another
size or storage, truncated or corrupted images are refused."""
import numpy as np
import pytest

from conftest import sphere_case

pytestmark = pytest.mark.gpu

DRAIN = dict(G=-5.0, rhos=0.223144, tau=1.0, inlet_width=3, outlet_width=1,
             rho_inlet=0.17, rho_outlet=1.90, rho_shift=1.0)
SHAPE = (48, 40, 36)


def _lattice(capi, fluid, rho, storage, kernel):
    lat = capi.Lattice(fluid.shape, storage=storage)
    lat.set_step_kernel(kernel)
    lat.set_params(capi.default_params(**DRAIN))
    lat.upload(fluid, rho)
    lat.initialize()
    return lat


def _state(lat, step):
    lat.iterate(step, 1, write_velocity=True)
    return lat.field("rho"), lat.field("f"), lat.field("velocity")


@pytest.mark.parametrize("storage,kernel", [(0, 0), (0, 6), (1, 0), (1, 6),
                                            (2, 0), (0, 2)])
@pytest.mark.parametrize("k", [7, 10])
def test_resume_is_bit_identical(storage, kernel, k):
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(SHAPE, seed=3 + k, rmin=2.0, rmax=4.5,
                             porosity=0.55, rho0=1.9, amp=0.05)
    a = _lattice(capi, fluid, rho, storage, kernel)
    a.iterate(0, k)
    image = a.checkpoint(k)
    a.iterate(k, 9)
    want = _state(a, k + 9)
    b = capi.Lattice(SHAPE, storage=storage)
    b.set_step_kernel(kernel)
    assert b.restore(image) == k
    b.iterate(k, 9)
    got = _state(b, k + 9)
    for u, v in zip(got, want):
        assert np.array_equal(u, v)
    a.close()
    b.close()


def test_resume_through_a_file(tmp_path):
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(SHAPE, seed=1, rmin=2.0, rmax=4.5, porosity=0.55,
                             rho0=1.9, amp=0.05)
    a = _lattice(capi, fluid, rho, 1, capi.KERNEL_BAND)
    a.iterate(0, 5)
    path = str(tmp_path / "lattice.ckpt")
    a.write_checkpoint(path, 5)
    a.iterate(5, 6)
    want = a.field("f")
    b = capi.Lattice(SHAPE, storage=1)
    assert b.read_checkpoint(path) == 5
    b.iterate(5, 6)
    assert np.array_equal(b.field("f"), want)
    a.close()
    b.close()


def test_refuses_foreign_truncated_and_corrupted_images():
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(SHAPE, seed=2, rmin=2.0, rmax=4.5, porosity=0.55,
                             rho0=1.9, amp=0.05)
    a = _lattice(capi, fluid, rho, 0, 0)
    a.iterate(0, 3)
    image = a.checkpoint(3)
    for lat in (capi.Lattice((48, 40, 35)), capi.Lattice(SHAPE, storage=1)):
        with pytest.raises(capi.MlbmError):
            lat.restore(image)
        lat.close()
    b = capi.Lattice(SHAPE)
    with pytest.raises(capi.MlbmError):
        b.restore(image[: len(image) - 1])
    bad = image.copy()
    bad[len(bad) // 2] ^= 1
    with pytest.raises(capi.MlbmError, match="corrupted"):
        b.restore(bad)
    bad = image.copy()
    bad[0] ^= 1
    with pytest.raises(capi.MlbmError, match="not a checkpoint"):
        b.restore(bad)
    with pytest.raises(capi.MlbmError):
        capi.Lattice(SHAPE).checkpoint(0)  # not initialised
    a.close()
    b.close()


@pytest.mark.parametrize("storage", [0, 1])
def test_batch_domain_preempted_and_resumed(storage):
    """Preemption in a batch: a domain saved (Lattice.checkpoint of the
    domain's lattice) and removed after 7 steps, the batch advanced without
    it, then the image admitted again (mlbm_batch_add_checkpoint) and run 9
    more steps, ends bit-identical to the domain run 16 steps alone."""
    from multiphase_lbm_b200 import batch, capi
    shapes = [(40, 32, 24), (48, 40, 36)]
    cases = [sphere_case(s, seed=20 + i, rmin=2.0, rmax=4.5, porosity=0.55,
                         rho0=1.9, amp=0.05) for i, s in enumerate(shapes)]
    p = capi.default_params(**DRAIN)
    b = batch.Batch(storage)
    ids = [b.add(fl, rho, p) for fl, rho in cases]
    b.iterate(7)
    b.synchronize()
    image = b.lattice(ids[0]).checkpoint(b.domain_step(ids[0]))
    b.remove(ids[0])
    b.iterate(5)
    did = b.add_checkpoint(image)
    assert b.domain_step(did) == 7
    b.iterate(9)
    b.synchronize()
    got = b.lattice(did).field("f")
    alone = _lattice(capi, cases[0][0], cases[0][1], storage, 0)
    alone.iterate(0, 16)
    assert np.array_equal(got, alone.field("f"))
    other = _lattice(capi, cases[1][0], cases[1][1], storage, 0)
    other.iterate(0, 21)
    assert np.array_equal(b.lattice(ids[1]).field("f"), other.field("f"))
    b.close()


@pytest.mark.parametrize("storage", [0, 1])
def test_long_run_saved_resumed_and_reallocated(storage):
    """Hundreds of steps, statistics read on the way, the lattice saved,
    destroyed and resumed in a fresh lattice (whose buffers reuse the freed
    memory), then hundreds more steps: bit-identical to the uninterrupted
    run -- the serving flow on single lattices."""
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(SHAPE, seed=9, rmin=2.0, rmax=4.5, porosity=0.55,
                             rho0=1.9, amp=0.05)
    a = _lattice(capi, fluid, rho, storage, 0)
    a.iterate(0, 400)
    a.stats()
    image = a.checkpoint(400)
    a.close()
    b = capi.Lattice(SHAPE, storage=storage)
    assert b.restore(image) == 400
    b.iterate(400, 300)
    b.stats()
    b.iterate(700, 300)
    ref = _lattice(capi, fluid, rho, storage, 0)
    ref.iterate(0, 1000)
    assert np.array_equal(b.field("f"), ref.field("f"))
    b.close()
    ref.close()
