"""TEI primitives with the reference's structure, on torch + libquax_b200.

The reference (quax/integrals/tei.py:12-181, 336-346, 403-411) defines JAX
primitives ``eri`` and ``eri_deriv`` whose JVP treats the incoming tangent as an
integer derivative-order vector (valid for the one-hot tangents jacfwd feeds),
plus a batching rule that loops over the one-hot rows.  JAX is not installed on
this image, so the same rules are given here as plain methods on torch tensors:

    eri(geom)                       -> (n,n,n,n) device tensor
    eri_deriv(geom, deriv_vec)      -> (n,n,n,n) slice, mode 'core' (precomputed
                                       first-derivative tensor, tei.py:31-34) or
                                       'f12' (computed per call, tei.py:152-154)
    eri_jvp((geom,), (tangent,))    -> (eri, eri_deriv(geom, tangent)) (tei.py:336-340)
    eri_deriv_jvp(...)              -> deriv_vec + tangent selects the next order
    eri_deriv_batch(geom, rows)     -> stacked slices for a batch of one-hot rows

``geom`` is a placeholder exactly as in the reference: the integrals are evaluated
at the geometry the engine was built with.  The differentiable entry point that
does use the geometry is :class:`EriEnergy` / :func:`two_electron_gradient`,
which contract the adjoint kernel instead of materialising 3N x n^4 tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from ..utils import get_deriv_vec_idx, how_many_derivs
from . import _lib
from .engine import EriEngine


class TEI:
    def __init__(self, basis, max_deriv_order: int = 0, mode: str = "core", ints_tol: float = 1.0e-14,
                 engine: EriEngine | None = None):
        self.engine = engine if engine is not None else EriEngine(basis, ints_tol)
        self.natom = self.engine.natom
        self.nbf = self.engine.nbf
        self.mode = mode
        # mode "disk" (tei.py:157-181): derivative slices are read from
        # eri_derivs.(h5|npz) written by libint_interface.compute_2e_deriv_disk
        if mode not in ("core", "f12", "disk"):
            raise ValueError(f"unknown mode {mode}")
        self.eri_derivatives = []
        if mode == "core" and max_deriv_order > 0:
            # tei.py:29-34: one tensor of unique derivatives per order
            top = _lib.load().qx_max_deriv_order()
            if max_deriv_order > top:
                raise NotImplementedError(f"precomputed derivative tensors of order {max_deriv_order} (this build: {top})")
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
            from .libint_interface import read_dataset

            n = self.nbf
            data = read_dataset("eri_derivs", f"eri_{n}_{n}_{n}_{n}_deriv{order}")
            return torch.from_numpy(np.ascontiguousarray(data[..., get_deriv_vec_idx(dv)])).to(self.engine.device)
        return self.engine.eri_deriv(dv)

    def eri_jvp(self, primals, tangents):
        (geom,) = primals
        return self.eri(geom), self.eri_deriv(geom, tangents[0])

    def eri_deriv_jvp(self, primals, tangents):
        geom, deriv_vec = primals
        dv = np.asarray(deriv_vec, dtype=int) + np.asarray(tangents[0], dtype=int)
        return self.eri_deriv(geom, deriv_vec), self.eri_deriv(geom, dv)

    def eri_deriv_batch(self, geom, deriv_batch):
        return torch.stack([self.eri_deriv(geom, row) for row in deriv_batch]), 0


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
