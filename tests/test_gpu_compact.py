"""The kernels over the compact (fluid-only) population layout.

COMPACT runs the two passes of the dense kernels over the compact layout and
BAND does both in one launch with two population buffers; both must match
the dense two-pass kernels bit for bit, and the reference's kernels (the
oracle) to the FP32 parity bar: density within 1e-5 relative pointwise,
populations and velocity within 1e-5 relative to their largest value, over
the first 100 steps.
"""
import numpy as np
import pytest

import oracle
from conftest import pointwise_rel_err, rel_err, sphere_case

pytestmark = pytest.mark.gpu

DRAIN = dict(G=-5.0, rhos=0.223144, tau=1.0, inlet_width=3, outlet_width=1,
             rho_inlet=0.17, rho_outlet=1.90)


def _lattice(capi, shape, fluid, rho, kernel, storage=0, **kw):
    lat = capi.Lattice(shape, storage=storage)
    lat.set_step_kernel(kernel)
    lat.set_params(capi.default_params(**kw))
    lat.upload(fluid, rho)
    lat.initialize()
    return lat


KINDS = [3, 6]  # KERNEL_COMPACT, KERNEL_BAND


@pytest.mark.parametrize("kind", KINDS)
def test_compact_matches_oracle_drainage_100_steps(kind):
    from multiphase_lbm_b200 import capi
    shape = (64, 48, 40)
    fluid, rho = sphere_case(shape, seed=11, rmin=3.0, rmax=6.0, porosity=0.55,
                             rho0=1.9, amp=0.02)
    lat = _lattice(capi, shape, fluid, rho, kind, **DRAIN)
    port = oracle.Port(rho, fluid, oracle.make_params(**DRAIN))
    m = fluid.astype(bool)
    step = 0
    for n in (1, 9, 89):
        lat.iterate(step, n)
        port.step(step, n)
        step += n
        e = pointwise_rel_err(lat.field("rho"), port.get("rho"), m)
        assert e <= 1e-5, f"step {step}: rho {e:.3e}"
        e = rel_err(lat.field("f"), port.get("f"), m)
        assert e <= 1e-5, f"step {step}: populations {e:.3e}"
    lat.iterate(step, 1, write_velocity=True)
    port.step(step, 1)
    e = rel_err(lat.field("velocity")[m], port.get("velocity")[m])
    assert e <= 1e-5, f"velocity {e:.3e}"


@pytest.mark.parametrize("storage", [0, 1])
@pytest.mark.parametrize("shape", [(40, 32, 24), (33, 5, 7), (70, 3, 2),
                                   (300, 6, 6), (1, 9, 8)])
def test_compact_two_pass_bit_identical(shape, storage):
    """Same loads, same arithmetic: the compact two-pass step equals the
    dense two-pass step bit for bit (drainage slabs, velocity output)."""
    from multiphase_lbm_b200 import capi
    fluid, rho = sphere_case(shape, seed=sum(shape) + storage, rmin=1.5,
                             rmax=3.5, porosity=0.6, rho0=1.5, amp=0.3)
    kw = dict(G=-5.0, rhos=0.223144, tau=1.0, rho_shift=1.0)
    if shape[0] >= 8:
        kw.update(inlet_width=2, outlet_width=1, rho_inlet=0.17, rho_outlet=1.9)
    outs = []
    for kind in (capi.KERNEL_COMPACT, capi.KERNEL_TWO_PASS):
        lat = _lattice(capi, shape, fluid, rho, kind, storage=storage, **kw)
        lat.iterate(0, 20)
        lat.iterate(20, 1, write_velocity=True)
        outs.append((lat.field("rho"), lat.field("f"), lat.field("velocity"),
                     lat.field("psi")))
    for u, v in zip(*outs):
        assert np.array_equal(u, v)


def test_fresh_lattices_first_steps_bit_identical():
    """The compact step kernels overlap their prologue with the kernel before
    them (programmatic dependent launch) and read the node table before
    they wait; the table is built earlier in the stream than that kernel.
    Lattices created, stepped and destroyed one after another (their buffers
    reuse the freed memory of the previous ones) give, from their very first
    step, the bits of the dense two-pass step."""
    from multiphase_lbm_b200 import capi
    shape = (40, 36, 28)
    kw = dict(DRAIN, rho_shift=1.0)
    cases = [sphere_case(shape, seed=40 + i, rmin=2.0, rmax=4.0, porosity=0.6,
                         rho0=1.2, amp=0.6) for i in range(3)]
    want = []
    for fluid, rho in cases:
        ref = _lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **kw)
        ref.iterate(0, 3)
        want.append(ref.field("f"))
        ref.close()
    for rep in range(8):
        fluid, rho = cases[rep % 3]
        lat = _lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT, **kw)
        lat.iterate(0, 3)
        assert np.array_equal(lat.field("f"), want[rep % 3]), rep
        lat.close()


def test_overlapped_steps_random_runs_against_dense_kernels():
    """Small lattices (where a step kernel does not fill the GPU), random run
    lengths with statistics read between them and one save / destroy /
    restore into a fresh lattice, under the launch overlap of the compact
    kernels: the final state equals the dense two-pass kernels' (launched
    without overlap) bit for bit, cycle after cycle."""
    from multiphase_lbm_b200 import capi, host
    rng = np.random.default_rng(2024)
    kw = dict(DRAIN, rho_shift=1.0)
    for cycle in range(40):
        shape = tuple(int(v) for v in rng.choice([16, 24, 32, 40], 3))
        storage = int(rng.integers(0, 2))
        fluid, _ = host.generate_packing(shape, 2.0, 5.0,
                                         float(rng.uniform(0.4, 0.7)),
                                         int(rng.integers(1 << 30)))
        rho = (1.0 + rng.uniform(-0.6, 0.6, shape)).astype(np.float32)
        plan = [int(v) for v in rng.integers(1, 80, int(rng.integers(1, 4)))]
        save_at = int(rng.integers(0, len(plan)))
        finals = []
        for kernel in (capi.KERNEL_COMPACT, capi.KERNEL_TWO_PASS):
            lat = _lattice(capi, shape, fluid, rho, kernel, storage=storage, **kw)
            step = 0
            for i, n in enumerate(plan):
                lat.iterate(step, n)
                step += n
                lat.stats()
                if i == save_at:
                    image = lat.checkpoint(step)
                    lat.close()
                    lat = capi.Lattice(shape, storage=storage)
                    lat.set_step_kernel(kernel)
                    assert lat.restore(image) == step
            finals.append(lat.field("f"))
            lat.close()
        assert np.array_equal(finals[0], finals[1]), (cycle, shape, storage, plan)


def test_steps_captured_in_a_cuda_graph():
    """mlbm_iterate captured into a CUDA graph on the lattice's stream (the
    step kernels are then launched without overlap) and replayed: the same
    bits as the steps run in stream order."""
    import torch

    from multiphase_lbm_b200 import capi
    shape = (40, 36, 28)
    fluid, rho = sphere_case(shape, seed=77, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=1.2, amp=0.6)
    kw = dict(DRAIN, rho_shift=1.0)
    stream = torch.cuda.Stream()
    a = _lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT, **kw)
    torch.cuda.synchronize()  # set-up ran on the legacy stream
    a.set_stream(stream.cuda_stream)
    a.iterate(0, 2)  # enters the fluid-only layout (allocations) first
    a.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        a.iterate(2, 2)  # two steps: the AA phase is the same after a replay
    for _ in range(5):
        graph.replay()
    torch.cuda.synchronize()
    b = _lattice(capi, shape, fluid, rho, capi.KERNEL_COMPACT, **kw)
    b.iterate(0, 12)
    assert np.array_equal(a.field("f"), b.field("f"))
    del graph
    a.close()
    b.close()


def test_kernel_switching_keeps_the_state():
    """band -> two-pass -> compact -> band -> two-pass, against two-pass
    throughout: the state moves between the layouts and buffers exactly."""
    from multiphase_lbm_b200 import capi
    shape = (40, 24, 20)
    fluid, rho = sphere_case(shape, seed=2, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=1.9, amp=0.02)
    a = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
    b = _lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **DRAIN)
    step = 0
    for kind in (capi.KERNEL_BAND, capi.KERNEL_TWO_PASS, capi.KERNEL_COMPACT,
                 capi.KERNEL_BAND, capi.KERNEL_TWO_PASS):
        a.set_step_kernel(kind)
        a.iterate(step, 15)
        b.iterate(step, 15)
        step += 15
    assert np.array_equal(a.field("rho"), b.field("rho"))
    assert np.array_equal(a.field("f"), b.field("f"))


def test_band_shape_autotune():
    from multiphase_lbm_b200 import capi
    shape = (64, 32, 32)
    fluid, rho = sphere_case(shape, seed=5, rmin=2.0, rmax=5.0, porosity=0.5,
                             rho0=1.9, amp=0.02)
    a = _lattice(capi, shape, fluid, rho, capi.KERNEL_BAND, **DRAIN)
    b = _lattice(capi, shape, fluid, rho, capi.KERNEL_TWO_PASS, **DRAIN)
    rows, planes, done = a.autotune(0, trial_steps=2)
    assert rows in (2, 4, 6, 8) and planes in (8, 16, 24, 32, 48) and done > 0
    b.iterate(0, done)
    a.set_band_shape(3, 5)
    a.iterate(done, 10)
    b.iterate(done, 10)
    assert np.array_equal(a.field("rho"), b.field("rho"))


def test_compact_kernels_reject_what_they_cannot_run():
    from multiphase_lbm_b200 import capi
    lat = capi.Lattice((16, 16, 16), storage=capi.STORE_F64)
    for kind in (capi.KERNEL_COMPACT, capi.KERNEL_BAND):
        with pytest.raises(capi.MlbmError):
            lat.set_step_kernel(kind)
    assert lat.step_kernel == capi.KERNEL_TWO_PASS       # AUTO on FP64
    for retired in (1, 4, 5, 7):
        with pytest.raises(capi.MlbmError):
            lat.set_step_kernel(retired)
    lat = capi.Lattice((16, 3, 16))
    lat.set_step_kernel(capi.KERNEL_COMPACT)
    lat.set_step_kernel(capi.KERNEL_BAND)


@pytest.mark.parametrize("storage", [0, 1])
def test_compact_large_rows_bit_identical(storage):
    """Rows of ~100 fluid nodes (a block of 256-512 nodes spans a few rows,
    as in the benchmark lattice): the compact two-pass step equals the dense
    two-pass step bit for bit, drainage slabs and velocity output included."""
    from multiphase_lbm_b200 import capi
    shape = (200, 96, 80)
    fluid, rho = sphere_case(shape, seed=77, rmin=4.0, rmax=10.0,
                             porosity=0.5, rho0=1.9, amp=0.05)
    kw = dict(DRAIN, rho_shift=1.0)
    outs = []
    for kind in (capi.KERNEL_COMPACT, capi.KERNEL_TWO_PASS):
        lat = _lattice(capi, shape, fluid, rho, kind, storage=storage, **kw)
        lat.iterate(0, 30)
        lat.iterate(30, 1, write_velocity=True)
        lat.synchronize()
        outs.append((lat.field("rho"), lat.field("f"), lat.field("velocity")))
    for u, v in zip(*outs):
        assert np.array_equal(u, v)
