"""The C ABI library loads without a GPU and exports every function that
include/*.h declares; the Python bindings cover them."""
import os
import re

import pytest

from multiphase_lbm_b200 import batch, capi, driver, host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = ["mlbm.h", "mlbm_host.h", "mlbm_driver.h", "mlbm_compat.h",
           "mlbm_batch.h"]


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)
    skip = {"if", "defined", "sizeof", "return"}
    return sorted({n for n in names if n not in skip and not n.startswith("__")})


@pytest.mark.parametrize("header", HEADERS)
def test_every_declared_function_is_exported(header):
    lib = capi.lib()
    missing = [n for n in _declared(header) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_abi():
    bound = {n for n, _, _ in capi.SIGNATURES}
    bound |= {n for n, _, _ in host.HOST_SIGNATURES}
    bound |= {n for n, _, _ in driver.DRIVER_SIGNATURES}
    bound |= {n for n, _, _ in batch.BATCH_SIGNATURES}
    for header in ("mlbm.h", "mlbm_host.h", "mlbm_driver.h", "mlbm_batch.h"):
        for name in _declared(header):
            assert name in bound, name


def test_status_strings_and_tables():
    L = capi.lib()
    assert L.mlbm_abi_version() == 1
    assert L.mlbm_status_string(5) == b"device wait timed out"
    import ctypes as C
    import numpy as np
    import oracle
    e = np.zeros(57, np.int32)
    w = np.zeros(19, np.float32)
    L.mlbm_d3q19(e.ctypes.data, w.ctypes.data)
    e = e.reshape(19, 3)
    assert (e[:, 0] == oracle.EX).all() and (e[:, 1] == oracle.EY).all()
    assert (e[:, 2] == oracle.EZ).all()
    assert np.allclose(w, oracle.T)


def test_errors_without_a_gpu_are_statuses():
    """No GPU here: creating a lattice returns MLBM_ERR_CUDA, never exits."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(capi.MlbmError) as e:
        capi.Lattice((8, 8, 8))
    assert e.value.status == 2
    with pytest.raises(capi.MlbmError) as e:
        capi.Lattice((0, 8, 8))
    assert e.value.status in (1, 2)
