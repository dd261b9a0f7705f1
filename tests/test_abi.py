"""The C-ABI library loads and exports every entry point the public header
declares; without a GPU the device entry points fail with a status code
instead of crashing or blocking."""
import ctypes as C

import pytest


def test_exports_match_header():
    import cfdfs
    L = cfdfs.lib()
    names = cfdfs.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.cfd_abi_version() == 1


def test_default_options():
    import cfdfs
    o = cfdfs.default_options()
    assert o.precision == cfdfs.FP64 and o.cg_rtol == 1e-8 and o.cg_maxit == 1000 and o.cg_warm == 0


def test_null_arguments_are_rejected():
    import cfdfs
    L = cfdfs.lib()
    assert L.cfd_step0(None) == cfdfs.CFD_E_BADARG
    assert L.cfd_run(None, 1, None) == cfdfs.CFD_E_BADARG
    assert L.cfd_load_inp(None, b"x") == cfdfs.CFD_E_BADARG
    assert L.cfdh_load(None, b"x", None, 0) == cfdfs.CFD_E_BADARG


def test_create_without_gpu_returns_status():
    import torch
    import cfdfs
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = cfdfs.lib().cfd_create(C.byref(h), 0)
    assert rc == cfdfs.CFD_E_CUDA and not h.value
