"""ctypes binding of ``libpfc_b200.so`` (the C ABI of ``include/pfc_b200.h``).

The shared library is built in-tree by :mod:`pfc_models_b200.build` and must
sit next to this file ($PFC_B200_LIB may name another build of it, for A/B
timing). There is no fallback: if the library is missing or a CUDA device is
absent, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfc_b200.so")

PFC_OK, PFC_E_ARG, PFC_E_CUDA, PFC_E_NAN, PFC_E_TIMEOUT, PFC_E_STATE, PFC_E_NOMEM = range(7)
MODEL_STD, MODEL_LOG = 0, 1
FP64_PLAIN, FP32_MIXED = 0, 1
FIELD_N, FIELD_MU, FIELD_LOCAL_MU, FIELD_LOCAL_N, FIELD_NONLIN_MU = range(5)
FIELD_OF_CURRENT = 0x100
SPEC_N_HAT, SPEC_N_HAT_NOW = 0, 1
FLAG_GENERIC_ONLY, FLAG_NO_GRAPHS, FLAG_PDL = 1, 2, 4
FLAG_PDL_COL = 128
FLAG_NO_ONE_CTA = 8
FLAG_PACKED = 16
FLAG_EXTV = 32
FLAG_TMA = 64
PATH_MIXED_RADIX, PATH_POW2, PATH_ONE_CTA, PATH_FAST_MIXED = 0, 1, 2, 3
STATUS_NONFINITE = 1
STATUS_TIMEOUT = 2


EE_PACKED = 0x80
PACKED_NONE, PACKED_BOTH, PACKED_ROW, PACKED_COL = 0, 1, 2, 3


def flag_variant(ee_row=0, ee_col=0, row_tile=0, col_cta=0, pdl=0, packed=0, tma=0, generic=0):
    """problem.flags bits selecting a step-kernel variant (PFC_FLAG_ROW_EE & co.).
    `packed`: 0 one-lane kernels, 1 the two-lane packed FP32 kernels on both passes,
    2 on the row pass only, 3 on the column pass only (then ee_* of a packed pass count
    values per lane). `pdl`: 1 both step kernels as programmatic dependent launches, 2 the
    column kernel only. `generic`: the run-time mixed-radix kernels instead."""
    cc = {0: 0, 1: 1, 2: 2, 4: 3}[int(col_cta)]
    packed = int(packed)
    er = int(ee_row) | (EE_PACKED if packed == PACKED_ROW else 0)
    ec = int(ee_col) | (EE_PACKED if packed == PACKED_COL else 0)
    return (er << 8) | (ec << 16) | (int(row_tile) << 24) | (cc << 29) | \
        (FLAG_PDL if pdl == 1 else FLAG_PDL_COL if pdl == 2 else 0) | \
        (FLAG_PACKED if packed == PACKED_BOTH else 0) | (FLAG_TMA if tma else 0) | \
        (FLAG_GENERIC_ONLY if generic else 0)

# every symbol include/pfc_b200.h declares, with (restype, argtypes)
_vp, _i32, _i64, _dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "pfc_abi_version": (ctypes.c_int, []),
    "pfc_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "pfc_plan_create": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "pfc_plan_destroy": (ctypes.c_int, [_vp]),
    "pfc_set_state": (ctypes.c_int, [_vp, _vp, _vp]),
    "pfc_get_state": (ctypes.c_int, [_vp, _vp, _vp]),
    "pfc_step": (ctypes.c_int, [_vp, _i64, _vp]),
    "pfc_step_timed": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(_dbl), ctypes.POINTER(_dbl), _vp]),
    "pfc_reduce": (ctypes.c_int, [_vp, _vp, _vp]),
    "pfc_get_field": (ctypes.c_int, [_vp, ctypes.c_int, _dbl, _vp, _vp]),
    "pfc_get_spectrum": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "pfc_get_coefficients": (ctypes.c_int, [_vp, _vp, _vp]),
    "pfc_status": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "pfc_plan_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64)]),
    "pfc_launch_count": (_i64, [_vp]),
    "pfc_plan_variant": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "pfc_plan_path": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "pfc_field_mean_noalloc": (ctypes.c_int, [_vp, _i64, _vp, _vp]),
    "pfc_batch_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, ctypes.POINTER(_vp)]),
    "pfc_batch_step": (ctypes.c_int, [_vp, _i64, _vp]),
    "pfc_batch_destroy": (ctypes.c_int, [_vp]),
    "pfc_batch_launch_count": (_i64, [_vp]),
    "pfc_batch_classes": (ctypes.c_int, [_vp]),
    "pfc_queue_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, ctypes.POINTER(_vp)]),
    "pfc_queue_step": (ctypes.c_int, [_vp, _i64, _vp]),
    "pfc_queue_status": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "pfc_queue_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "pfc_queue_launch_count": (_i64, [_vp]),
    "pfc_queue_destroy": (ctypes.c_int, [_vp]),
    "pfc_test_queue_wait": (ctypes.c_int, [_vp, _i32, _i64]),
    "pfc_locate_vacancies": (ctypes.c_int, [_vp, _i32, _i32, _dbl, _dbl, _vp, _i32, _vp, _vp]),
    "pfc_diagnose_modes": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _dbl, _vp, _vp]),
    "pfc_frozen_moments": (ctypes.c_int, [_vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _dbl, _vp, _vp]),
    "pfc_defect_screen": (ctypes.c_int, [_vp, _vp, _vp, _dbl, _dbl, _vp, _vp]),
    "pfc_set_potential": (ctypes.c_int, [_vp, _vp, _vp]),
    "pfc_extv_state": (ctypes.c_int, [_vp, ctypes.POINTER(_dbl)]),
    "pfc_extv_set_tolerances": (ctypes.c_int, [_vp, _dbl, _dbl]),
    "pfc_test_tma_wait": (ctypes.c_int, [_vp, _i32, _i32]),
}


class PfcProblem(ctypes.Structure):
    """Mirror of ``pfc_problem`` in include/pfc_b200.h."""
    _fields_ = [
        ("nx", _i32), ("ny", _i32), ("model", _i32), ("precision", _i32),
        ("lx", _dbl), ("ly", _dbl),
        ("gamma", _dbl), ("beta", _dbl), ("q0", _dbl), ("epsilon", _dbl), ("g", _dbl), ("dt", _dbl),
        ("small_z_tol", _dbl), ("min_phi", _dbl),
        ("clamp_log", _i32), ("flags", _i32),
    ]


class PfcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[pfc error {code}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def load(path: str | None = None):
    """Load the library once; raise if it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or os.environ.get("PFC_B200_LIB") or LIB_PATH
        if not os.path.exists(p):
            raise ImportError(f"{p} is not built: run `python -m pfc_models_b200.build` "
                              "(there is no CPU fallback)")
        lib = ctypes.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().pfc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != PFC_OK:
        raise PfcError(rc, last_error())
