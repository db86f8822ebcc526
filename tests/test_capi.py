"""The C-ABI library loads and exports every entry point include/pfc_b200.h declares.

No compute call is made here (these tests run without a GPU): only argument
validation that returns before any CUDA call.
"""
import ctypes
import os
import re

from tests.conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "pfc_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pfc_[a-z0-9_]+)\s*\(", src)))


def test_header_matches_binding():
    from pfc_models_b200 import _lib
    assert _declared() == sorted(_lib.SIGNATURES)


def test_library_exports_all_symbols(built_lib):
    lib = ctypes.CDLL(built_lib)
    for name in _declared():
        assert hasattr(lib, name), f"{name} not exported"


def test_abi_version_and_errors(built_lib):
    from pfc_models_b200 import _lib
    lib = _lib.load(built_lib)
    assert lib.pfc_abi_version() == 1
    prob = _lib.PfcProblem(nx=5, ny=8, model=0, precision=0, lx=1.0, ly=1.0, dt=0.1)
    h = ctypes.c_void_p()
    rc = lib.pfc_plan_create(ctypes.byref(prob), ctypes.byref(h))
    assert rc == _lib.PFC_E_ARG and not h.value
    assert "nx must be even" in _lib.last_error()
    prob = _lib.PfcProblem(nx=34, ny=8, model=0, precision=0, lx=1.0, ly=1.0, dt=0.1)  # 17 is prime
    assert lib.pfc_plan_create(ctypes.byref(prob), ctypes.byref(h)) == _lib.PFC_E_ARG
    assert "prime factor" in _lib.last_error()
    prob = _lib.PfcProblem(nx=8, ny=8, model=7, precision=0, lx=1.0, ly=1.0, dt=0.1)
    assert lib.pfc_plan_create(ctypes.byref(prob), ctypes.byref(h)) == _lib.PFC_E_ARG
    assert lib.pfc_step(None, 1, None) == _lib.PFC_E_ARG
    assert lib.pfc_launch_count(None) == 0
