"""The C ABI library loads and exports every symbol include/quax_b200.h declares,
and rejects invalid input on the host before any device work (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "quax_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from quax_b200.integrals import _lib

    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_build_info():
    from quax_b200.integrals import _lib

    lib = _lib.load()
    assert lib.qx_max_l() == 3  # f shells
    assert lib.qx_max_deriv_order() == 4
    assert lib.qx_num_classes() == 55  # canonical classes up to (ff|ff)


def _init(lib, _lib, coords, exps, tol=1e-12, l=(0,), nprim=(1,), atom=(0,)):
    l = np.asarray(l, dtype=np.int32)
    nprim = np.asarray(nprim, dtype=np.int32)
    atom = np.asarray(atom, dtype=np.int32)
    coefs = np.ones_like(exps)
    h = ctypes.c_void_p()
    return lib.qx_initialize(len(coords) // 3, _lib.dptr(coords), len(l), _lib.iptr(l), _lib.iptr(nprim),
                             _lib.iptr(atom), _lib.dptr(exps), _lib.dptr(coefs), 0, tol, ctypes.byref(h))


@pytest.mark.parametrize("case", ["nan_coord", "bad_tol", "pure", "empty"])
def test_initialize_rejects_invalid_input_on_host(case):
    from quax_b200.integrals import _lib

    lib = _lib.load()
    coords = np.zeros(3)
    exps = np.array([1.0])
    if case == "nan_coord":
        coords[1] = np.nan
        assert _init(lib, _lib, coords, exps) == _lib.QX_E_INVALID
        assert b"coordinate" in lib.qx_last_error()
    elif case == "bad_tol":
        assert _init(lib, _lib, coords, exps, tol=-1.0) == _lib.QX_E_INVALID
    elif case == "pure":
        h = ctypes.c_void_p()
        l = np.zeros(1, dtype=np.int32)
        rc = lib.qx_initialize(1, _lib.dptr(coords), 1, _lib.iptr(l), _lib.iptr(np.ones(1, np.int32)),
                               _lib.iptr(l), _lib.dptr(exps), _lib.dptr(exps), 1, 1e-12, ctypes.byref(h))
        assert rc == _lib.QX_E_UNSUPPORTED
    else:
        h = ctypes.c_void_p()
        assert lib.qx_initialize(0, None, 0, None, None, None, None, None, 0, 1e-12, ctypes.byref(h)) == _lib.QX_E_INVALID


def test_check_maps_codes_to_exceptions():
    from quax_b200.integrals import _lib

    with pytest.raises(ValueError):
        _lib.check(_lib.QX_E_INVALID, "x")
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.QX_E_UNSUPPORTED, "x")
    with pytest.raises(MemoryError):
        _lib.check(_lib.QX_E_NOMEM, "x")
    with pytest.raises(_lib.QuaxError):
        _lib.check(_lib.QX_E_CUDA, "x")
