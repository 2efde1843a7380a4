"""Shared fixtures.  ``-m gpu`` tests need a CUDA device; everything else runs
on the CPU.  Native libraries are built in-tree on first use (a machine that
receives the tree with them built uses them as they are)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ensure_built():
    import oracle
    from multiphase_lbm_b200 import build as pkg_build
    if not os.path.exists(pkg_build.LIB):
        pkg_build.build()
    if not os.path.exists(os.path.join(oracle.HERE, "liboracle_f32.so")):
        oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    return torch.cuda.is_available()


def random_case(shape, seed=0, solid_frac=0.25, rho0=0.7, amp=0.01):
    """Seeded random fluid mask and density around rho0 (reference layout)."""
    rng = np.random.default_rng(seed)
    fluid = (rng.random(shape) >= solid_frac).astype(np.uint8)
    rho = (rho0 + rng.uniform(-amp, amp, shape)).astype(np.float32)
    return fluid, rho


def sphere_case(shape, seed=0, rmin=2.5, rmax=7.5, porosity=0.5, rho0=0.7,
                amp=0.01):
    """Seeded sphere packing (libmlbm's generator) and density."""
    from multiphase_lbm_b200 import host
    fluid, _ = host.generate_packing(shape, rmin, rmax, porosity, seed)
    rng = np.random.default_rng(seed + 1000)
    rho = (rho0 + rng.uniform(-amp, amp, shape)).astype(np.float32)
    return fluid, rho


def rel_err(a, b, mask=None):
    """max |a - b| / max |b| over the masked entries."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def pointwise_rel_err(a, b, mask=None):
    """max_k |a_k - b_k| / |b_k| over the masked entries."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    return float((np.abs(a - b) / np.maximum(np.abs(b), 1e-30)).max())
