"""ctypes binding of libquax_b200.so (the C ABI declared in include/quax_b200.h).

The library is built in-tree by quax_b200.build.  There is no CPU fallback: if the
shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libquax_b200.so")

QX_OK = 0
QX_E_INVALID = -1
QX_E_CUDA = -2
QX_E_UNSUPPORTED = -3
QX_E_NOMEM = -4
QX_E_DEVICE = -5

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); every symbol of include/quax_b200.h
SIGNATURES = {
    "qx_last_error": (C.c_char_p, []),
    "qx_max_deriv_order": (C.c_int, []),
    "qx_max_l": (C.c_int, []),
    "qx_initialize": (
        C.c_int,
        [C.c_int, _dp, C.c_int, _ip, _ip, _ip, _dp, _dp, C.c_int, C.c_double, C.POINTER(_vp)],
    ),
    "qx_finalize": (C.c_int, [_vp]),
    "qx_nbf": (C.c_int, [_vp]),
    "qx_natom": (C.c_int, [_vp]),
    "qx_nshell": (C.c_int, [_vp]),
    "qx_unique_quartets": (C.c_longlong, [_vp]),
    "qx_unique_size": (C.c_longlong, [_vp]),
    "qx_schwarz": (C.c_int, [_vp, _dp, _dp]),
    "qx_compute_2e_int": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "qx_eri_unique": (C.c_int, [_vp, _vp, _vp]),
    "qx_eri_deriv_core": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp]),
    "qx_compute_2e_deriv": (C.c_int, [_vp, _ip, C.c_int, _vp, C.c_int, _vp]),
    "qx_grad_adjoint": (C.c_int, [_vp, _vp, C.c_double, C.c_double, _vp, C.c_int, _vp]),
    "qx_jk": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp]),
    "qx_num_classes": (C.c_int, []),
    "qx_class_info": (
        C.c_int,
        [_vp, C.c_int, _ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), _dp, _dp],
    ),
    "qx_eri_unique_class": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "qx_grad_adjoint_class": (C.c_int, [_vp, C.c_int, _vp, C.c_double, C.c_double, _vp, _vp]),
    "qx_autotune": (C.c_int, [_vp, C.c_int, _vp]),
    "qx_set_charges": (C.c_int, [_vp, _vp]),
    "qx_jk_screened": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, _vp]),
    "qx_oei": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "qx_oei_deriv_core": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
    "qx_grad_adjoint_jvp": (C.c_int, [_vp, _vp, C.c_double, C.c_double, _vp, _vp, C.c_int, _vp]),
    "qx_set_shard": (C.c_int, [_vp, C.c_int, C.c_int]),
    "qx_set_precision": (C.c_int, [_vp, C.c_double]),
    "qx_precision_split": (C.c_longlong, [_vp, C.c_int]),
    "qx_partition_costs": (C.c_int, [_vp, C.c_longlong, C.c_int, _vp]),
    "qx_engine_config": (C.c_int, [_vp, C.c_int, _vp]),
    "qx_set_engine": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "qx_class_quartets": (C.c_int, [_vp, C.c_int, _ip]),
    "qx_set_wait_limit": (C.c_int, [_vp, C.c_int]),
    "qx_deriv_tile": (C.c_int, [_vp, C.c_int, C.c_longlong, C.c_longlong, C.c_int, _vp, C.c_longlong, _vp]),
    "qx_gamma_tile": (C.c_int, [_vp, C.c_int, C.c_longlong, C.c_longlong, C.c_int, _vp, C.c_double, C.c_double, _vp,
                                _vp]),
    "qx_cart2sph_block": (C.c_int, [_vp, _vp, _ip, C.c_longlong, _dp, _vp]),
    "qx_release_scratch": (C.c_int, [_vp]),
    "qx_compute_2e_int_noalloc": (
        C.c_int,
        [C.c_int, _dp, C.c_int, _ip, _ip, _ip, _dp, _dp, C.c_double, _vp, _vp],
    ),
}

_LIB = None


class QuaxError(RuntimeError):
    pass


def load():
    """Load the library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise QuaxError(f"{LIB_PATH} is missing: run quax_b200.build.build() (no CPU fallback exists)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(rc: int, what: str = "") -> int:
    if rc >= 0:
        return rc
    msg = load().qx_last_error().decode()
    if rc == QX_E_INVALID:
        raise ValueError(f"{what}: {msg}")
    if rc == QX_E_UNSUPPORTED:
        raise NotImplementedError(f"{what}: {msg}")
    if rc == QX_E_NOMEM:
        raise MemoryError(f"{what}: {msg}")
    raise QuaxError(f"{what}: {msg} (code {rc})")


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)
