"""Generate the golden fixtures in this directory from the REFERENCE ITSELF.

Every output stored here was produced by the reference's own code -- its
kernels, device functions and host driver compiled for the CPU
(``oracle/_ref/libref_<size>.so``, built by ``oracle/build_ref.py`` from the
reference sources) -- on seeded synthetic inputs.  The fixtures let the tests
pin the oracle and the CUDA path on machines where the reference sources are
absent.

Run from the repository root:  ``python tests/golden/make_golden.py``
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

SC = dict(G=-6.0, rhos=0.182322, tau=1.0)


def random_case(shape, seed, solid_frac=0.25, rho0=0.7, amp=0.01):
    rng = np.random.default_rng(seed)
    fluid = (rng.random(shape) >= solid_frac).astype(np.uint8)
    rho = (rho0 + rng.uniform(-amp, amp, shape)).astype(np.float32)
    return fluid, rho


def run_case(name, shape, fluid, rho, params, checkpoints, step_kw=None):
    step_kw = step_kw or {}
    ref = oracle.Reference(shape)
    ref.setup(rho, fluid, oracle.make_params(**params))
    out = {"fluid": fluid, "rho0": rho}
    step = 0
    for cp in checkpoints:
        ref.step(step, cp - step, **step_kw)
        step = cp
        out[f"rho_{cp}"] = ref.get("rho")
    out[f"f_{checkpoints[-1]}"] = ref.get("f")
    out[f"force_{checkpoints[-1]}"] = ref.get("force")
    meta = dict(params)
    meta.update(step_kw)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                        meta=np.array(repr(meta)),
                        checkpoints=np.array(checkpoints), **out)
    print("wrote", name)


def voxel_case():
    """Masks from the reference driver's read_positions / place_sphere /
    generate_solids tokens and its rand() density initialisation."""
    from multiphase_lbm_b200 import host
    shape = (40, 40, 40)
    _, spheres = host.generate_packing(shape, 2.5, 7.5, 0.5, seed=11)
    ref = oracle.Reference(shape)
    with tempfile.TemporaryDirectory() as td:
        pos = os.path.join(td, "positions.txt")
        host.write_positions(pos, spheres)
        cmd = os.path.join(td, "input.txt")
        with open(cmd, "w") as fh:
            fh.write("rho0 0.7\nIniPerturbRate 0.0285714\nresize\n"
                     "resolution 1\n"
                     f"read_positions {pos}\n"
                     "place_sphere 3.5 35.25 20.0 4.75\n"
                     "generate_solids 3 2.0 4.0 0 40 0 40 0 40\n")
        rho, fluid, sn, info = ref.driver_read(cmd)
    spheres_txt = np.array([float(f"{v:.9g}") for v in spheres.ravel()],
                           np.float32).reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "voxel_40.npz"),
                        spheres=spheres_txt, fluid=fluid, solid_number=sn,
                        rho=rho, packing_density=info["packing_density"],
                        solid_count=info["solid_count"])
    print("wrote voxel_40")


def main():
    sh = (16, 12, 10)
    f, r = random_case(sh, 1)
    run_case("periodic_16x12x10", sh, f, r, SC, [1, 10, 100])
    sh = (24, 20, 18)
    f, _ = random_case(sh, 2, solid_frac=0.3)
    r = np.full(sh, 2.0, np.float32)
    run_case("drainage_24x20x18", sh, f, r,
             dict(SC, inlet_width=3, outlet_width=1, rho_inlet=0.10,
                  rho_outlet=1.95), [1, 10, 100])
    sh = (16, 12, 10)
    f, r = random_case(sh, 3, rho0=0.2, amp=0.05)
    run_case("inject_cs_16x12x10", sh, f, r,
             dict(G=-1.0, tau=1.0, carn_star=1, T_Tc=0.7, rhos=0.35,
                  rho_increment=0.005, rho_inject_period=3,
                  inject_position=0.5, inject_density=1),
             [1, 10, 60], step_kw=dict(inject_type=1, reverse=1))
    voxel_case()


if __name__ == "__main__":
    main()
