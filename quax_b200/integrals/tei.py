"""TEI primitives with the reference's structure, on torch + libquax_b200.

The reference (quax/integrals/tei.py:12-181, 336-346, 403-411) defines JAX
primitives ``eri`` and ``eri_deriv`` whose JVP treats the incoming tangent as an
integer derivative-order vector (valid for the one-hot tangents jacfwd feeds),
plus a batching rule that loops over the one-hot rows.  JAX is not installed on
this image, so the same rules are given here as plain methods on torch tensors,
with the reference's signatures:

    TEI(basis1, basis2, basis3, basis4, xyz_path, max_deriv_order, options, mode)
                                    (tei.py:14; basis objects with .nbf() or basis
                                    names; the geometry read from xyz_path)
    eri(geom)                       -> (n,n,n,n) device tensor
    eri_deriv(geom, deriv_vec)      -> (n,n,n,n) slice: mode 'core' (precomputed
                                       tensors of every order <= max_deriv_order,
                                       tei.py:29-34), 'f12' (computed per call,
                                       tei.py:152-154) or 'disk' (eri_derivs, else
                                       eri_partials, tei.py:157-181)
    eri_jvp((geom,), (tangent,))    -> (eri, eri_deriv(geom, tangent)) (tei.py:336-340)
    eri_deriv_jvp(...)              -> deriv_vec + tangent selects the next order
    eri_deriv_batch(batched_args, batch_dims)
                                    -> (stacked slices of the one-hot rows, 0)
                                       (tei.py:403-411)

Like the reference, the integrals come from the ``libint_interface`` module's
state (set by its initialize(), quax/methods/ints.py:20): a TEI built while that
module is initialised uses its engine.  Otherwise the TEI initialises it from
xyz_path and the basis (a name, or an in-memory Basis whose shells sit on the
xyz file's atoms).  ``geom`` is a placeholder exactly as in the reference: the
integrals are evaluated at the geometry the engine was built with.  The
differentiable entry point that does use the geometry is
:func:`two_electron_energy`, whose backward pass is the adjoint kernel.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from ..basis import Basis, Molecule
from ..utils import get_deriv_vec_idx, how_many_derivs
from . import _lib
from .engine import EriEngine


def _nbf(basis) -> int:
    """nbf() of a basis object (the reference passes psi4 BasisSet objects)."""
    return int(basis.nbf()) if callable(getattr(basis, "nbf", None)) else int(basis.nbf)


class TEI:
    def __init__(self, basis1, basis2=None, basis3=None, basis4=None, xyz_path=None, max_deriv_order: int = 0,
                 options=None, mode: str = "core", *, ints_tol: float | None = None, engine: EriEngine | None = None):
        from . import libint_interface as li

        options = dict(options or {})
        tol = ints_tol if ints_tol is not None else float(options.get("ints_tolerance", 1.0e-14))
        if mode not in ("core", "f12", "disk"):
            raise ValueError(f"unknown mode {mode}")
        if engine is None:
            if xyz_path is not None:
                # the reference's form: natoms from the xyz file, nbf from the bases
                mol = Molecule.from_xyz(xyz_path, units="angstrom")
                bases = [b for b in (basis1, basis2, basis3, basis4) if b is not None]
                if len({_nbf(b) if not isinstance(b, str) else b for b in bases}) > 1:
                    raise NotImplementedError("the ERI path uses one basis for all four centres")
                if li.is_initialized():
                    engine = li.engine()
                elif isinstance(basis1, str):
                    li.initialize(xyz_path, basis1, basis1, basis1, basis1, tol)
                    engine = li.engine()
                else:
                    li.initialize_basis(basis1.with_coords(mol.coords), tol, charges=mol.Z)
                    engine = li.engine()
                if engine.natom != mol.natom:
                    raise ValueError(f"{xyz_path} has {mol.natom} atoms, the integral engine {engine.natom}")
            else:
                # in-memory basis (this package's own callers)
                if not isinstance(basis1, Basis):
                    raise ValueError("TEI needs xyz_path, or an in-memory Basis as basis1")
                engine = EriEngine(basis1, tol)
        self.engine = engine
        self.natom = engine.natom
        self.nbf = self.nbf1 = self.nbf2 = self.nbf3 = self.nbf4 = engine.nbf
        if basis1 is not None and not isinstance(basis1, str) and _nbf(basis1) != self.nbf:
            raise ValueError(f"basis has {_nbf(basis1)} functions, the integral engine {self.nbf}")
        self.mode = mode
        self.eri_derivatives = []
        if mode == "core" and max_deriv_order > 0:
            # tei.py:29-34: one tensor of unique derivatives per order
            top = _lib.load().qx_max_deriv_order()
            if max_deriv_order > top:
                raise NotImplementedError(f"precomputed derivative tensors of order {max_deriv_order} (this library: {top})")
            for k in range(1, max_deriv_order + 1):
                d = self.engine.eri_deriv_core(k)
                assert d.shape[0] == how_many_derivs(self.natom, k)
                self.eri_derivatives.append(d)

    def eri(self, geom=None) -> torch.Tensor:
        return self.engine.eri()

    def eri_deriv(self, geom, deriv_vec) -> torch.Tensor:
        dv = np.asarray(deriv_vec.cpu() if torch.is_tensor(deriv_vec) else deriv_vec, dtype=int).reshape(-1)
        order = int(dv.sum())
        if order == 0:
            return self.eri(geom)
        if self.mode == "core":
            if order > len(self.eri_derivatives):
                raise NotImplementedError(f"order {order} derivatives were not precomputed")
            return self.eri_derivatives[order - 1][get_deriv_vec_idx(dv)]
        if self.mode == "disk":
            return self._read_disk(order, get_deriv_vec_idx(dv))
        return self.engine.eri_deriv(dv)

    def _read_disk(self, order: int, idx: int) -> torch.Tensor:
        """tei.py:157-181: the full tensors eri_derivs (datasets eri_n_n_n_n_deriv<k>,
        derivative index last), else the per-slice file eri_partials (datasets
        eri_n_n_n_n_deriv<k>_<idx>); .h5 where h5py is present, .npz otherwise."""
        from .libint_interface import read_dataset

        n = self.nbf
        base = f"eri_{n}_{n}_{n}_{n}_deriv{order}"
        if os.path.exists("eri_derivs.h5") or os.path.exists("eri_derivs.npz"):
            data = read_dataset("eri_derivs", base)
        elif os.path.exists("eri_partials.h5") or os.path.exists("eri_partials.npz"):
            data = read_dataset("eri_partials", f"{base}_{idx}")
        else:
            raise FileNotFoundError("ERI derivatives not found on disk")
        if data.ndim == 5:
            data = data[..., idx]
        elif data.ndim != 4:
            raise ValueError("Something went wrong reading integral derivative file")
        return torch.from_numpy(np.ascontiguousarray(data)).to(self.engine.device)

    def eri_jvp(self, primals, tangents):
        (geom,) = primals
        return self.eri(geom), self.eri_deriv(geom, tangents[0])

    def eri_deriv_jvp(self, primals, tangents):
        geom, deriv_vec = primals
        dv = np.asarray(deriv_vec, dtype=int) + np.asarray(tangents[0], dtype=int)
        return self.eri_deriv(geom, deriv_vec), self.eri_deriv(geom, dv)

    def eri_deriv_batch(self, batched_args, batch_dims):
        """tei.py:403-411: evaluate every row of the batched deriv_vec argument and
        stack the slices along a new leading axis, which is the output batch axis."""
        geom_batch, deriv_batch = batched_args
        return torch.stack([self.eri_deriv(geom_batch, row) for row in deriv_batch]), 0


class _EriEnergy(torch.autograd.Function):
    """E_2e = sum_ijkl Gamma_ijkl (ij|kl) with Gamma = cj D_ij D_kl + ck D_ik D_jl.

    Forward returns E_2e (the dense tensor is formed only for small n); backward
    returns dE/dgeom through the adjoint kernel (never the 3N x n^4 tensor)."""

    @staticmethod
    def forward(ctx, geom, D, engine, cj, ck):
        G = engine.eri()
        Dd = D.to(G.device)
        E = cj * torch.einsum("ij,kl,ijkl->", Dd, Dd, G) + ck * torch.einsum("ik,jl,ijkl->", Dd, Dd, G)
        ctx.engine, ctx.cj, ctx.ck = engine, cj, ck
        ctx.geom_device, ctx.geom_dtype = geom.device, geom.dtype
        ctx.save_for_backward(D)
        return E

    @staticmethod
    def backward(ctx, gE):
        (D,) = ctx.saved_tensors
        g = ctx.engine.grad_adjoint(D, ctx.cj, ctx.ck)
        g = (gE.to(g.device) * g).to(device=ctx.geom_device, dtype=ctx.geom_dtype)
        return g.reshape(-1), None, None, None, None


def two_electron_energy(geom, D, engine: EriEngine, cj=1.0, ck=-0.5):
    """Differentiable two-electron energy; its gradient w.r.t. geom uses the adjoint."""
    return _EriEnergy.apply(geom, D, engine, cj, ck)


def two_electron_gradient(D, engine: EriEngine, cj=1.0, ck=-0.5):
    """sum_ijkl Gamma_ijkl d(ij|kl)/dR, (3N,) device tensor."""
    return engine.grad_adjoint(D, cj, ck)
