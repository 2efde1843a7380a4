"""Batched domains: every domain advanced in a batch is bit-identical to the
same domain advanced alone (alone vs in the mix), with and without CUDA
graphs, across tuning changes, and with domains joining and leaving."""
import numpy as np
import pytest

from conftest import sphere_case

pytestmark = pytest.mark.gpu


def _params(capi, i, shape):
    return capi.default_params(G=-6.0, tau=1.0, rhos=0.1 + 0.02 * i,
                               inlet_width=max(1, shape[0] // 16),
                               outlet_width=1, rho_inlet=0.1 + 0.01 * i,
                               rho_outlet=1.9)


def _alone(capi, shape, fluid, rho, params, storage, steps):
    # FP32 / FP16 batches run the compact kernels, FP64 batches the dense
    # two-pass kernels; both are bit-identical to the dense two-pass step
    lat = capi.Lattice(shape, storage=storage)
    lat.set_step_kernel(capi.KERNEL_TWO_PASS)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    lat.iterate(0, steps)
    out = lat.field("rho"), lat.field("f")
    lat.close()
    return out


SHAPES = [(32, 48, 16), (48, 32, 32), (64, 16, 48), (40, 40, 40), (33, 17, 9)]


@pytest.mark.parametrize("storage", [0, 1, 2])
def test_batch_equals_alone(storage):
    from multiphase_lbm_b200 import batch, capi
    cases = []
    for i, sh in enumerate(SHAPES):
        fl, rho = sphere_case(sh, seed=10 + i, rmin=2.0, rmax=4.0,
                              porosity=0.6, rho0=2.0 - 0.2 * i, amp=0.01)
        cases.append((sh, fl, rho, _params(capi, i, sh)))
    b = batch.Batch(storage)
    ids = [b.add(fl, rho, p) for sh, fl, rho, p in cases]
    b.iterate(13)
    b.set_tuning(2, 8, 3, 0, graphs=True)
    b.iterate(17)   # two graph replays + direct steps
    b.synchronize()
    for did, (sh, fl, rho, p) in zip(ids, cases):
        r_b, f_b = b.lattice(did).field("rho"), b.lattice(did).field("f")
        r_a, f_a = _alone(capi, sh, fl, rho, p, storage, 30)
        assert np.array_equal(r_b, r_a), sh
        assert np.array_equal(f_b, f_a), sh
        assert b.domain_step(did) == 30
    b.close()


def test_batch_join_and_leave_midway():
    from multiphase_lbm_b200 import batch, capi
    b = batch.Batch(0)
    a_sh, c_sh = (40, 24, 20), (24, 40, 12)
    fa, ra = sphere_case(a_sh, seed=1, rmin=2, rmax=4, porosity=0.6)
    fc, rc = sphere_case(c_sh, seed=2, rmin=2, rmax=4, porosity=0.6)
    pa, pc = _params(capi, 0, a_sh), _params(capi, 3, c_sh)
    ia = b.add(fa, ra, pa)
    b.iterate(11)                     # odd: the next domain joins in phase 1
    ic = b.add(fc, rc, pc)
    b.iterate(20)
    b.remove(ia)
    b.iterate(5)
    b.synchronize()
    r_c = b.lattice(ic).field("rho")
    assert np.array_equal(r_c, _alone(capi, c_sh, fc, rc, pc, 0, 25)[0])
    assert b.domain_step(ic) == 25 and b.count() == 1
    b.close()


def test_batch_autotune_runs_and_keeps_results():
    from multiphase_lbm_b200 import batch, capi
    sh = (48, 48, 48)
    fl, rho = sphere_case(sh, seed=5, rmin=2, rmax=5, porosity=0.55)
    p = _params(capi, 1, sh)
    b = batch.Batch(0)
    did = b.add(fl, rho, p)
    choice = b.autotune(2)
    steps = b.domain_step(did)
    b.iterate(10)
    b.synchronize()
    assert set(choice) == {"rows_density", "rows_update", "planes",
                           "blocks_per_sm"}
    r = b.lattice(did).field("rho")
    assert np.array_equal(r, _alone(capi, sh, fl, rho, p, 0, steps + 10)[0])
    b.close()
