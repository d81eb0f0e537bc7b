"""The C ABI library loads on a CPU-only machine and exports every entry point
include/lbm_b200.h declares; without a GPU, creation fails cleanly."""
import ctypes
import re

import numpy as np
import pytest

from lbm_b200 import capi


def declared_functions():
    text = open(capi.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(capi.SIGNATURES)


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_create_rejects_bad_descriptor():
    d = capi.LbmDesc()
    d.lattice = 20
    h = ctypes.c_void_p()
    rc = capi.lib().lbm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == capi.LBM_ERR_ARGUMENT
    assert b"lattice" in capi.lib().lbm_last_error(None)


def test_reference_mode_requires_d3q19():
    d = capi.LbmDesc()
    d.lattice, d.bc_mode, d.tau = 27, capi.BC_REFERENCE, 0.8
    h = ctypes.c_void_p()
    rc = capi.lib().lbm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == capi.LBM_ERR_ARGUMENT
    assert b"D3Q19" in capi.lib().lbm_last_error(None)


def test_null_handle_calls_fail_cleanly():
    L = capi.lib()
    assert L.lbm_step(None, 1) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_destroy(None) == capi.LBM_ERR_ARGUMENT
    assert L.lbm_last_error(None)


def test_create_without_gpu_reports_no_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lbm_b200 import Engine
    topo = {"coords": np.array([[0, 0, 0], [0, 0, 1]]), "kind": np.zeros(2, np.uint8),
            "inlet": np.zeros(0), "inlet_normal": np.zeros(3), "wall": np.zeros(0),
            "nearwall": np.zeros(0), "nearwall_normal": np.zeros((0, 3))}
    with pytest.raises(capi.LbmError) as ei:
        Engine(topo, tau=0.8)
    assert ei.value.code == capi.LBM_ERR_NO_DEVICE
