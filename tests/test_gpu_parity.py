"""Parity of the CUDA time step (through the C ABI) with the oracle.

The oracle is ``oracle/mlbm_oracle.c`` (a C restatement that reproduces the
reference's own kernels bit for bit, see test_oracle_pin.py) on the same
seeded inputs.  Tolerances (the parity bar of the FP32 drop-in):
  * FP32 storage: density within 1e-5 relative (pointwise over fluid nodes)
    and populations / velocity within 1e-5 relative to their largest value,
    over the first 100 steps;
  * FP64 storage against the FP64 oracle: 1e-12;
  * FP16 storage (populations stored as half(f - t_i rho0)): density within
    2e-3 relative over 100 steps.
"""
import numpy as np
import pytest

import oracle
from conftest import pointwise_rel_err, random_case, rel_err, sphere_case

pytestmark = pytest.mark.gpu

SC_PARAMS = dict(G=-6.0, rhos=0.182322, tau=1.0)
# the default kernel (the compact single-pass step where supported) and the
# two-pass kernels
KERNELS = [0, 2]


def _pair(shape, fluid, rho, storage=0, f64_oracle=False, kernel=0, **kw):
    from multiphase_lbm_b200 import capi
    p = capi.default_params(**kw)
    op = oracle.make_params(**{k: v for k, v in kw.items()
                               if k not in ("rho_shift",)})
    lat = capi.Lattice(shape, storage=storage)
    lat.set_step_kernel(kernel)
    lat.set_params(p)
    lat.upload(fluid, rho)
    lat.initialize()
    port = oracle.Port(rho, fluid, op, f64=f64_oracle)
    return lat, port


def _compare(lat, port, fluid, tol_rho, tol_f, label, f64=False):
    m = fluid.astype(bool)
    r_gpu = lat.field("rho", f64=f64)
    r_cpu = port.get("rho")
    e_rho = pointwise_rel_err(r_gpu, r_cpu, m)
    e_f = rel_err(lat.field("f", f64=f64), port.get("f"), m)
    assert e_rho <= tol_rho, f"{label}: rho rel err {e_rho:.3e} > {tol_rho}"
    assert e_f <= tol_f, f"{label}: populations rel err {e_f:.3e} > {tol_f}"
    return e_rho, e_f


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("shape", [(24, 20, 18), (33, 7, 5), (64, 9, 3)])
def test_periodic_random_mask_fp32(shape, kernel):
    fluid, rho = random_case(shape, seed=sum(shape))
    lat, port = _pair(shape, fluid, rho, kernel=kernel, **SC_PARAMS)
    step = 0
    for n in (1, 9, 90):
        lat.iterate(step, n)
        port.step(step, n)
        step += n
        _compare(lat, port, fluid, 1e-5, 1e-5, f"{shape} step {step}")


@pytest.mark.parametrize("kernel", KERNELS)
def test_sphere_packing_64_fp32_100_steps(kernel):
    """Phase separation on a 64^3 packing (G=-6, G_ads=-1 -> rhos=0.182322,
    rho 0.70+-0.01)."""
    shape = (64, 64, 64)
    fluid, rho = sphere_case(shape, seed=7)
    lat, port = _pair(shape, fluid, rho, kernel=kernel, **SC_PARAMS)
    lat.iterate(0, 99)
    port.step(0, 99)
    lat.iterate(99, 1, write_velocity=True)
    port.step(99, 1)
    _compare(lat, port, fluid, 1e-5, 1e-5, "64^3 step 100")
    # velocity u = (sum f e + tau F)/rho of the last step
    m = fluid.astype(bool)
    e = rel_err(lat.field("velocity")[m], port.get("velocity")[m])
    assert e <= 1e-5, f"velocity rel err {e:.3e}"


@pytest.mark.parametrize("kernel", KERNELS)
def test_drainage_boundary_fp32(kernel):
    shape = (40, 24, 20)
    fluid, rho = sphere_case(shape, seed=3, rmin=2.0, rmax=4.0, porosity=0.6,
                             rho0=2.0, amp=0.0)
    kw = dict(SC_PARAMS, inlet_width=3, outlet_width=1, rho_inlet=0.10,
              rho_outlet=1.95)
    lat, port = _pair(shape, fluid, rho, kernel=kernel, **kw)
    step = 0
    for n in (1, 9, 90):
        lat.iterate(step, n)
        port.step(step, n)
        step += n
        _compare(lat, port, fluid, 1e-5, 1e-5, f"drainage step {step}")


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("inject_type,reverse", [(0, 1), (1, 1), (2, -1)])
def test_injection_fp32(inject_type, reverse, kernel):
    shape = (24, 20, 18)
    fluid, rho = random_case(shape, seed=11, rho0=0.5, amp=0.3)
    kw = dict(SC_PARAMS, rho_increment=0.01, rho_inject_period=3,
              inject_position=0.5, inject_density=1)
    lat, port = _pair(shape, fluid, rho, kernel=kernel, **kw)
    lat.iterate(0, 30, reverse=reverse, inject_type=inject_type)
    port.step(0, 30, reverse=reverse, inject_type=inject_type)
    _compare(lat, port, fluid, 1e-5, 1e-5, f"inject {inject_type}")


def test_carnahan_starling_fp32():
    shape = (24, 20, 18)
    fluid, rho = random_case(shape, seed=5, rho0=0.2, amp=0.05)
    kw = dict(tau=1.0, G=-1.0, carn_star=1, T_Tc=0.7, rhos=0.35)
    lat, port = _pair(shape, fluid, rho, **kw)
    lat.iterate(0, 50)
    port.step(0, 50)
    _compare(lat, port, fluid, 1e-5, 1e-5, "CS EOS")


def test_tau_not_one_fp32():
    shape = (24, 20, 18)
    fluid, rho = random_case(shape, seed=6)
    lat, port = _pair(shape, fluid, rho, G=-6.0, rhos=0.3, tau=0.8)
    lat.iterate(0, 60)
    port.step(0, 60)
    _compare(lat, port, fluid, 1e-5, 1e-5, "tau 0.8")


def test_fp64_storage_matches_fp64_oracle():
    shape = (24, 20, 18)
    fluid, rho = random_case(shape, seed=8)
    lat, port = _pair(shape, fluid, rho, storage=2, f64_oracle=True,
                      **SC_PARAMS)
    lat.iterate(0, 50)
    port.step(0, 50)
    _compare(lat, port, fluid, 1e-12, 1e-12, "fp64", f64=True)


def test_fp16_storage_close_to_fp64_oracle():
    shape = (32, 24, 20)
    fluid, rho = random_case(shape, seed=9, rho0=1.0, amp=0.05)
    lat, port = _pair(shape, fluid, rho, storage=1, f64_oracle=True,
                      rho_shift=1.0, **SC_PARAMS)
    lat.iterate(0, 100)
    port.step(0, 100)
    m = fluid.astype(bool)
    e = pointwise_rel_err(lat.field("rho"), port.get("rho"), m)
    assert e <= 2e-3, e


@pytest.mark.parametrize("kernel", KERNELS)
def test_all_fluid_and_all_solid_edges(kernel):
    shape = (16, 8, 8)
    rho = np.full(shape, 0.7, np.float32)
    for fl in (np.ones(shape, np.uint8), np.zeros(shape, np.uint8)):
        lat, port = _pair(shape, fl, rho, kernel=kernel, **SC_PARAMS)
        lat.iterate(0, 5)
        port.step(0, 5)
        if fl.any():
            _compare(lat, port, fl, 1e-6, 1e-6, "all fluid")
        else:
            r = lat.field("rho")
            assert np.all(r == np.float32(0.182322))


def test_determinism_bitwise():
    shape = (48, 40, 36)
    fluid, rho = sphere_case(shape, seed=21)
    outs = []
    for _ in range(2):
        lat, _port = _pair(shape, fluid, rho, **SC_PARAMS)
        lat.iterate(0, 40)
        outs.append((lat.field("rho"), lat.field("f")))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_phase_stats_match_oracle():
    shape = (40, 32, 24)
    fluid, rho = sphere_case(shape, seed=4, rho0=0.7, amp=0.01)
    lat, port = _pair(shape, fluid, rho, **SC_PARAMS)
    lat.iterate(0, 200)
    port.step(0, 200)
    s = lat.stats()
    o = port.phase_stats()
    assert s["n_fluid"] == int(o[0])
    # classification of a node whose rho sits within 1e-5 of a threshold may
    # differ; allow a handful of nodes
    assert abs(s["n_liquid"] - int(o[1])) <= 3
    assert abs(s["n_vapour"] - int(o[2])) <= 3
    assert abs(s["mass"] - o[7]) <= 1e-5 * o[7]
    assert abs(s["min_rho"] - o[8]) <= 1e-5 * abs(o[8]) + 1e-7
    assert abs(s["max_rho"] - o[9]) <= 1e-5 * abs(o[9])


def test_async_stats_equal_sync_stats_every_step():
    """mlbm_phase_stats_async, read one step later while the next step runs,
    gives exactly the statistics mlbm_phase_stats gives at that step."""
    import torch

    from multiphase_lbm_b200 import capi
    shape = (48, 40, 32)
    fluid, rho = sphere_case(shape, seed=6, rho0=0.7, amp=0.05)
    a, _ = _pair(shape, fluid, rho, **SC_PARAMS)
    b, _ = _pair(shape, fluid, rho, **SC_PARAMS)
    raw = [torch.zeros(capi.STATS_RAW_LEN, dtype=torch.float64).pin_memory().numpy()
           for _ in range(2)]
    ev = [torch.cuda.Event() for _ in range(2)]
    got, want = [], []
    for k in range(12):
        a.iterate(k, 1)
        a.stats_async(raw[k % 2])
        ev[k % 2].record()
        if k > 0:
            ev[(k - 1) % 2].synchronize()
            got.append(a.stats_from_raw(raw[(k - 1) % 2]))
        b.iterate(k, 1)
        want.append(b.stats())
    ev[11 % 2].synchronize()
    got.append(a.stats_from_raw(raw[11 % 2]))
    assert got == want


BULK_KEYS = ("n_fluid", "n_liquid", "n_vapour", "mass", "sum_rho_liquid",
             "sum_rho_vapour", "saturation", "avg_rho_liquid",
             "avg_rho_vapour", "min_rho", "max_rho")


@pytest.mark.parametrize("storage,kernel", [(0, 0), (1, 0), (2, 0), (0, 2)],
                         ids=["f32-auto", "f16-auto", "f64", "f32-dense"])
def test_bulk_stats_equal_the_full_statistics(storage, kernel):
    """mlbm_bulk_stats_async: its columns are bit-identical to
    mlbm_phase_stats on the same state (the fluid-list walk of the compact
    layout, the dense walk in FP32 and FP64), the columns it skips read 0,
    and a second call gives the same result.  The lattice has more fluid
    nodes than one wave of the fluid-list walk's blocks covers (~114 k on a
    B200), so its blocks take spans of several rounds."""
    import torch

    from multiphase_lbm_b200 import capi
    shape = (96, 80, 64)
    fluid, _ = sphere_case(shape, seed=8)
    # liquid, vapour and in-between nodes side by side in the initial state
    # (one step of streaming mixes them: after it no node is vapour); then
    # after one and two steps, the two AA phases
    rho = np.random.default_rng(8).uniform(0.02, 0.9, shape).astype(np.float32)
    lat, _ = _pair(shape, fluid, rho, storage=storage, kernel=kernel,
                   **SC_PARAMS)
    raw = torch.zeros(capi.STATS_RAW_LEN, dtype=torch.float64).pin_memory().numpy()
    for step in range(3):
        if step:
            lat.iterate(step, 1)
        lat.bulk_stats_async(raw)
        lat.synchronize()
        bulk = lat.stats_from_raw(raw)
        full = lat.stats()
        lat.bulk_stats_async(raw)
        lat.synchronize()
        assert lat.stats_from_raw(raw) == bulk
        assert full["n_liquid"] > 0 and (step or full["n_vapour"] > 0)
        for key in BULK_KEYS:
            assert bulk[key] == full[key], key
        for key in set(full) - set(BULK_KEYS):
            assert bulk[key] == 0, key
    lat.close()


def test_mass_conservation_periodic_full_size():
    """Periodic, no injection: total fluid mass is conserved (BGK and
    bounce-back conserve mass); FP64 reduction, 200^3, 20 steps."""
    shape = (200, 200, 200)
    fluid, rho = sphere_case(shape, seed=1, rmin=5, rmax=15, rho0=0.7)
    from multiphase_lbm_b200 import capi
    lat = capi.Lattice(shape)
    lat.set_params(capi.default_params(**SC_PARAMS))
    lat.upload(fluid, rho)
    lat.initialize()
    lat.iterate(0, 1)
    m0 = lat.stats()["mass"]
    lat.iterate(1, 20)
    m1 = lat.stats()["mass"]
    assert abs(m1 - m0) / m0 < 2e-6, (m0, m1)
