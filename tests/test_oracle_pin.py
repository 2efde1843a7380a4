"""Pin the oracle (oracle/mlbm_oracle.c) to the reference.

* against the golden fixtures in tests/golden/ -- outputs of the reference's
  own kernels (oracle/_ref, generated by tests/golden/make_golden.py): the
  FP32 restatement must reproduce them bit for bit;
* against the reference's own kernels run live (oracle/_ref), where that
  build exists, for more parameter combinations;
* the FP64 oracle against the FP32 one (same update, higher precision).
"""
import ast
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SC = dict(G=-6.0, rhos=0.182322, tau=1.0)


def _load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = ast.literal_eval(str(d["meta"]))
    return d, meta


@pytest.mark.parametrize("name", ["periodic_16x12x10", "drainage_24x20x18",
                                  "inject_cs_16x12x10"])
def test_port_reproduces_reference_golden_bitwise(name):
    d, meta = _load(name)
    step_kw = {k: meta.pop(k) for k in ("inject_type", "reverse") if k in meta}
    port = oracle.Port(d["rho0"], d["fluid"], oracle.make_params(**meta))
    step = 0
    cps = [int(c) for c in d["checkpoints"]]
    for cp in cps:
        port.step(step, cp - step, **step_kw)
        step = cp
        assert np.array_equal(port.get("rho"), d[f"rho_{cp}"]), (name, cp)
    assert np.array_equal(port.get("f"), d[f"f_{cps[-1]}"])
    assert np.array_equal(port.get("force"), d[f"force_{cps[-1]}"])


def _ref_or_skip(shape):
    if tuple(shape) not in oracle.reference_sizes():
        pytest.skip(f"oracle/_ref has no {shape} build")
    return oracle.Reference(shape)


@pytest.mark.parametrize("kw,step_kw", [
    (dict(SC), {}),
    (dict(SC, tau=0.7, rhos=0.4), {}),
    (dict(SC, rho_increment=0.01, rho_inject_period=2, inject_position=0.4,
          inject_density=1), dict(inject_type=0, reverse=-1)),
    (dict(SC, rho_increment=0.02, rho_inject_period=1, inject_density=1),
     dict(inject_type=2, reverse=1)),
    (dict(SC, inlet_width=2, outlet_width=2, rho_inlet=0.1, rho_outlet=1.9),
     {}),
    (dict(G=-1.0, carn_star=1, T_Tc=0.8, rhos=0.3, tau=1.2), {}),
])
def test_port_matches_reference_live(kw, step_kw):
    shape = (24, 20, 18)
    ref = _ref_or_skip(shape)
    rng = np.random.default_rng(42)
    fluid = (rng.random(shape) > 0.3).astype(np.uint8)
    rho0 = 0.25 if kw.get("carn_star") else 0.7
    rho = (rho0 + rng.uniform(-0.05, 0.05, shape)).astype(np.float32)
    p = oracle.make_params(**kw)
    ref.setup(rho, fluid, p)
    port = oracle.Port(rho, fluid, p)
    ref.step(0, 25, **step_kw)
    port.step(0, 25, **step_kw)
    for k in ("rho", "pressure", "psi", "force", "f"):
        assert np.array_equal(ref.get(k), port.get(k)), k


def test_fp64_oracle_tracks_fp32():
    d, meta = _load("periodic_16x12x10")
    p = oracle.make_params(**meta)
    a = oracle.Port(d["rho0"], d["fluid"], p)
    b = oracle.Port(d["rho0"], d["fluid"], p, f64=True)
    a.step(0, 100)
    b.step(0, 100)
    m = d["fluid"].astype(bool)
    ra, rb = a.get("rho")[m], b.get("rho")[m]
    assert np.abs(ra - rb).max() / np.abs(rb).max() < 1e-4


def test_oracle_tables_match_reference_model():
    # include/lbm_model.cuh:35-54 (weights sum to 1, opposite pairs i, i+9)
    assert abs(float(oracle.T.astype(np.float64).sum()) - 1.0) < 1e-7
    for i in range(1, 10):
        assert oracle.EX[i] == -oracle.EX[i + 9]
        assert oracle.EY[i] == -oracle.EY[i + 9]
        assert oracle.EZ[i] == -oracle.EZ[i + 9]
