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
        raise NotImplementedError(f"derivative order {deriv_order} (this library: {LIBINT2_MAX_DERIV_ORDER})")
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
        raise NotImplementedError(f"one-electron derivative order {order} (this library: 1)")
    return eng.oei_deriv(1)[k][int(np.argmax(dv))].reshape(-1).cpu().numpy()


def oei_deriv_core(deriv_order: int):
    if deriv_order != 1:
        raise NotImplementedError(f"one-electron derivative order {deriv_order} (this library: 1)")
    return [x.reshape(-1).cpu().numpy() for x in _engine().oei_deriv(1)]


def generate_multi_index_lookup(nparams: int, deriv_order: int):
    return _lookup(nparams, deriv_order)


# -- disk format (libint_interface.cc:1338-1567, 1811-2115; read by tei.py:157-181) ----
# The reference writes HDF5 files with one dataset per derivative order, named
# <type>_<nbf...>_deriv<k> and shaped (nbf..., nderiv) -- the derivative index last.
# h5py is optional here: with it the same .h5 files are written; without it the
# same datasets go to a NumPy archive of the same stem (.npz).
_DISK_LIMIT_GB = 50.0  # the reference asserts the same bound (libint_interface.cc:1819)


def _write_datasets(stem: str, datasets: dict) -> str:
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is not None:
        path = stem + ".h5"
        with h5py.File(path, "w") as f:
            for k, v in datasets.items():
                f.create_dataset(k, data=v)
    else:
        path = stem + ".npz"
        np.savez(path, **datasets)
    return path


def read_dataset(stem: str, name: str) -> np.ndarray:
    """One dataset of a file written by the *_deriv_disk functions (.h5 or .npz)."""
    import os

    if os.path.exists(stem + ".h5"):
        import h5py

        with h5py.File(stem + ".h5", "r") as f:
            return f[name][()]
    if os.path.exists(stem + ".npz"):
        with np.load(stem + ".npz") as z:
            return z[name]
    raise FileNotFoundError(f"{stem}.h5 / {stem}.npz not found")


def compute_2e_deriv_disk(type_: str, beta: float, max_deriv_order: int) -> str:
    """Write every ERI derivative tensor up to max_deriv_order to eri_derivs.(h5|npz):
    datasets eri_<n>_<n>_<n>_<n>_deriv<k>, shape (n, n, n, n, nderiv)."""
    _check_type(type_)
    eng = _engine()
    n = eng.nbf
    slices = sum(how_many_derivs(eng.natom, k) for k in range(1, max_deriv_order + 1))
    if n**4 * slices * 8e-9 >= _DISK_LIMIT_GB:
        raise ValueError(f"ERI derivative tensors need {n**4 * slices * 8e-9:.0f} GB (limit {_DISK_LIMIT_GB:.0f} GB)")
    if max_deriv_order > LIBINT2_MAX_DERIV_ORDER:
        raise NotImplementedError(f"derivative order {max_deriv_order} (this library: {LIBINT2_MAX_DERIV_ORDER})")
    data = {}
    for k in range(1, max_deriv_order + 1):
        d = eng.eri_deriv_core(k).cpu().numpy()
        data[f"eri_{n}_{n}_{n}_{n}_deriv{k}"] = np.ascontiguousarray(np.moveaxis(d, 0, -1))
    return _write_datasets("eri_derivs", data)


def compute_1e_deriv_disk(type_: str, max_deriv_order: int) -> str:
    """Write one-electron derivative tensors to oei_derivs.(h5|npz): datasets
    <type>_<n>_<n>_deriv<k>, shape (n, n, nderiv); first order in this library."""
    return _oei_disk([type_], max_deriv_order)


def oei_deriv_disk(max_deriv_order: int) -> str:
    """Overlap, kinetic and potential derivative tensors to oei_derivs.(h5|npz)."""
    return _oei_disk(list(_OEI_TYPES), max_deriv_order)


def _oei_disk(types, max_deriv_order: int) -> str:
    ks = [_oei_index(t) for t in types]
    if max_deriv_order != 1:
        raise NotImplementedError(f"one-electron derivative order {max_deriv_order} (this library: 1)")
    eng = _engine()
    n = eng.nbf
    d = eng.oei_deriv(1)
    data = {f"{_OEI_TYPES[k]}_{n}_{n}_deriv1": np.ascontiguousarray(np.moveaxis(d[k].cpu().numpy(), 0, -1))
            for k in ks}
    return _write_datasets("oei_derivs", data)


# -- device-resident variants (additions) -------------------------------------------
def compute_2e_int_device():
    """Dense (n,n,n,n) ERI tensor as a CUDA tensor (no host copy)."""
    return _engine().eri()


def eri_deriv_core_device(deriv_order: int = 1):
    return _engine().eri_deriv_core(deriv_order)


def engine() -> EriEngine:
    """The engine behind the module state (for the adjoint gradient and friends)."""
    return _engine()


def is_initialized() -> bool:
    """True between initialize() and finalize()."""
    return _state.get("engine") is not None
