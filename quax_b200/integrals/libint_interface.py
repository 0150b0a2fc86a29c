"""Drop-in for the ERI subset of the reference's pybind11 module ``libint_interface``.

Same names, argument meaning and error behaviour as
quax/integrals/libint_interface.cc:2784-2807, backed by libquax_b200.so:

    initialize(xyzfilename, basis1, basis2, basis3, basis4, ints_tol)   (:38-95)
    finalize()                                                          (:97-99)
    compute_2e_int("eri", beta)          -> 1-D float64 array of n^4     (:486-647)
    compute_2e_deriv("eri", beta, deriv_vec) -> 1-D array of n^4        (:1097-1335)
    eri_deriv_core(deriv_order)          -> 1-D array of nderiv*n^4      (:2582-2779)
    compute_1e_int(type)                 -> 1-D array of n^2 (overlap | kinetic | potential)  (:232-483)
    compute_1e_deriv(type, deriv_vec)    -> 1-D array of n^2 (first order)                   (:650-788)
    oei_deriv_core(deriv_order)          -> [overlap, kinetic, potential] nderiv*n^2 each    (:2403-2579)
    generate_multi_index_lookup(nparams, order) -> list of lists        (utils.h:158-172)
    LIBINT2_MAX_DERIV_ORDER                                              (:2806)

Like the reference, results come back as host arrays (copied off the device), the
module keeps global state between initialize() and finalize(), and an unknown
integral type raises ValueError (the reference's std::invalid_argument).  The
F12 operators and the HDF5 disk writers of the reference are not part of the ERI
path and raise NotImplementedError.  ``initialize_basis`` and the ``*_device``
variants are additions: they take an in-memory basis and return device tensors.
"""
from __future__ import annotations

import numpy as np

from ..basis import Basis, Molecule, build_basis
from ..utils import generate_multi_index_lookup as _lookup
from ..utils import how_many_derivs
from . import _lib
from .engine import EriEngine

_F12_TYPES = ("f12", "f12g12", "f12_squared", "f12_double_commutator")
_state = {"engine": None, "natom": 0}

LIBINT2_MAX_DERIV_ORDER = _lib.load().qx_max_deriv_order()


def initialize(xyzfilename: str, basis1: str, basis2: str, basis3: str, basis4: str, ints_tol: float) -> None:
    """Read the geometry (Angstrom xyz, as Libint's reader expects) and build the basis."""
    if not (basis1 == basis2 == basis3 == basis4):
        raise NotImplementedError("the ERI path uses one basis for all four centres (quax/methods/ints.py:20)")
    mol = Molecule.from_xyz(xyzfilename, units="angstrom")
    initialize_basis(build_basis(mol, basis1), ints_tol, charges=mol.Z)


def initialize_basis(basis: Basis, ints_tol: float, charges=None) -> None:
    """Same as initialize() for an in-memory basis (coordinates in bohr); the nuclear
    charges are needed only for the potential integrals."""
    finalize()
    _state["engine"] = EriEngine(basis, ints_tol)
    _state["natom"] = basis.natom
    if charges is not None:
        _state["engine"].set_charges(charges)


def finalize() -> None:
    eng = _state.get("engine")
    if eng is not None:
        eng.close()
    _state["engine"] = None


def _engine() -> EriEngine:
    eng = _state.get("engine")
    if eng is None:
        raise RuntimeError("libint_interface.initialize() must be called first")
    return eng


def _check_type(type_: str):
    if type_ in _F12_TYPES:
        raise NotImplementedError(f"operator '{type_}' is outside the ERI path of this library")
    if type_ != "eri":
        raise ValueError("type must be eri, f12, f12g12, f12_squared, or f12_double_commutator")


def compute_2e_int(type_: str, beta: float) -> np.ndarray:
    _check_type(type_)
    return _engine().eri().reshape(-1).cpu().numpy()


def compute_2e_deriv(type_: str, beta: float, deriv_vec) -> np.ndarray:
    _check_type(type_)
    eng = _engine()
    dv = np.asarray(deriv_vec, dtype=int).reshape(-1)
    if dv.size != 3 * eng.natom:
        # the reference asserts this (libint_interface.cc:1098)
        raise ValueError("Derivative vector incorrect size for this molecule.")
    return eng.eri_deriv(dv).reshape(-1).cpu().numpy()


def eri_deriv_core(deriv_order: int) -> np.ndarray:
    eng = _engine()
    if deriv_order > LIBINT2_MAX_DERIV_ORDER:
        raise NotImplementedError(f"derivative order {deriv_order} (this build: {LIBINT2_MAX_DERIV_ORDER})")
    out = eng.eri_deriv_core(deriv_order)
    assert out.shape[0] == how_many_derivs(eng.natom, deriv_order)
    return out.reshape(-1).cpu().numpy()


_OEI_TYPES = ("overlap", "kinetic", "potential")


def _oei_index(type_: str) -> int:
    if type_ not in _OEI_TYPES:
        raise ValueError("type must be overlap, kinetic, or potential")
    return _OEI_TYPES.index(type_)


def compute_1e_int(type_: str) -> np.ndarray:
    return _engine().oei()[_oei_index(type_)].reshape(-1).cpu().numpy()


def compute_1e_deriv(type_: str, deriv_vec) -> np.ndarray:
    k = _oei_index(type_)
    eng = _engine()
    dv = np.asarray(deriv_vec, dtype=int).reshape(-1)
    if dv.size != 3 * eng.natom:
        raise ValueError("Derivative vector incorrect size for this molecule.")
    order = int(dv.sum())
    if order == 0:
        return compute_1e_int(type_)
    if order != 1 or (dv < 0).any():
        raise NotImplementedError(f"one-electron derivative order {order} (this build: 1)")
    return eng.oei_deriv(1)[k][int(np.argmax(dv))].reshape(-1).cpu().numpy()


def oei_deriv_core(deriv_order: int):
    if deriv_order != 1:
        raise NotImplementedError(f"one-electron derivative order {deriv_order} (this build: 1)")
    return [x.reshape(-1).cpu().numpy() for x in _engine().oei_deriv(1)]


def generate_multi_index_lookup(nparams: int, deriv_order: int):
    return _lookup(nparams, deriv_order)


def compute_2e_deriv_disk(type_: str, beta: float, max_deriv_order: int):
    raise NotImplementedError("HDF5 disk mode (libint_interface.cc:1811-2115) is not part of this build")


# -- device-resident variants (additions) -------------------------------------------
def compute_2e_int_device():
    """Dense (n,n,n,n) ERI tensor as a CUDA tensor (no host copy)."""
    return _engine().eri()


def eri_deriv_core_device(deriv_order: int = 1):
    return _engine().eri_deriv_core(deriv_order)


def engine() -> EriEngine:
    """The engine behind the module state (for the adjoint gradient and friends)."""
    return _engine()
