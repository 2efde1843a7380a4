"""multiphase_lbm_b200 -- D3Q19 single-component Shan-Chen multiphase lattice
Boltzmann on NVIDIA B200 (sm_100a).

The product is ``libmlbm.so`` (CUDA kernels + host driver behind the C ABI of
``include/mlbm.h``, ``include/mlbm_host.h``, ``include/mlbm_compat.h``) and the
``mlbm`` command-line program.  This package holds their sources (``csrc/``),
the build recipe (``build.py``) and the ctypes bindings used from Python
(``capi``, ``host``)."""
from .capi import (Lattice, MlbmError, Params, Stats, default_params,  # noqa: F401
                   lattice_bytes, lib)

__all__ = ["Lattice", "MlbmError", "Params", "Stats", "default_params",
           "lattice_bytes", "lib"]
