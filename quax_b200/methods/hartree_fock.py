"""Restricted Hartree-Fock on the B200 integral path.

Mirrors the reference's RHF (quax/methods/hartree_fock.py:8-119): Cholesky
orthogonalisation (energy_utils.py:33-40), D = C_occ C_occ^T, F = H + 2J - K,
E = sum (F + H) o D + E_nuc.  Differences: J and K come from the direct kernel
(qx_jk) instead of contracting a dense G every iteration (hartree_fock.py:79-80),
the SCF uses DIIS extrapolation, and the geometric gradient is analytic,

    dE/dR = 2 sum D dH - 2 sum W dS + sum Gamma dG + dE_nuc,
    Gamma_ijkl = 2 D_ij D_kl - D_ik D_jl,  W = C_occ diag(eps_occ) C_occ^T,

with the two-electron term from the adjoint kernel (qx_grad_adjoint), so the
3N x n^4 derivative tensor is never formed (the reference forms it and
differentiates through every SCF iteration with jacfwd).  One-electron integrals
and their derivatives come from the GPU kernel (qx_oei, qx_oei_deriv_core).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from ..basis import Basis, Molecule
from ..integrals.engine import EriEngine
from ..oei import nuclear_repulsion


@dataclass
class RHFResult:
    energy: float
    C: torch.Tensor
    eps: torch.Tensor
    D: torch.Tensor
    iterations: int
    engine: EriEngine


def restricted_hartree_fock(mol: Molecule, basis: Basis, ints_tol: float = 1.0e-14, maxit: int = 100,
                            conv: float = 1.0e-10, engine: EriEngine | None = None, device: str = "cuda") -> RHFResult:
    dev = torch.device(device)
    eng = engine if engine is not None else EriEngine(basis, ints_tol, device=dev)
    eng.set_charges(mol.Z)
    St, T, V = eng.oei()
    H = T + V
    A = torch.linalg.inv(torch.linalg.cholesky(St)).T
    ndocc = mol.nelectron // 2
    Enuc = nuclear_repulsion(mol.Z, mol.coords)
    D = torch.zeros_like(H)
    F = H.clone()
    E_old = 0.0
    focks, errs = [], []
    it = 0
    for it in range(1, maxit + 1):
        Fp = A.T @ F @ A
        eps, C2 = torch.linalg.eigh(Fp)
        C = A @ C2
        Cocc = C[:, :ndocc]
        D = Cocc @ Cocc.T
        J, K = eng.jk(D)
        F = H + 2.0 * J - K
        E = float(torch.sum((F + H) * D)) + Enuc
        err = A.T @ (F @ D @ St - St @ D @ F) @ A
        focks.append(F)
        errs.append(err)
        if len(focks) > 8:
            focks.pop(0)
            errs.pop(0)
        if abs(E - E_old) < conv and float(torch.sqrt(torch.mean(err**2))) < conv:
            break
        E_old = E
        if len(focks) >= 2:  # Pulay DIIS on the commutator FDS - SDF
            m = len(focks)
            B = torch.empty((m + 1, m + 1), dtype=H.dtype, device=dev)
            B[-1, :] = -1.0
            B[:, -1] = -1.0
            B[-1, -1] = 0.0
            for i in range(m):
                for j in range(m):
                    B[i, j] = torch.sum(errs[i] * errs[j])
            rhs = torch.zeros(m + 1, dtype=H.dtype, device=dev)
            rhs[-1] = -1.0
            coef = torch.linalg.lstsq(B, rhs.unsqueeze(1)).solution.squeeze(1)
            F = sum(coef[i] * focks[i] for i in range(m))
    Fp = A.T @ (H + 2.0 * J - K) @ A
    eps, C2 = torch.linalg.eigh(Fp)
    C = A @ C2
    return RHFResult(E, C, eps, D, it, eng)


def rhf_gradient(mol: Molecule, basis: Basis, ints_tol: float = 1.0e-14, conv: float = 1.0e-11,
                 device: str = "cuda", result: RHFResult | None = None) -> tuple:
    """(energy, gradient (3N,)) of RHF; the ERI term by the adjoint kernel."""
    res = result if result is not None else restricted_hartree_fock(mol, basis, ints_tol, conv=conv, device=device)
    ndocc = mol.nelectron // 2
    Cocc = res.C[:, :ndocc]
    D = Cocc @ Cocc.T
    W = Cocc @ torch.diag(res.eps[:ndocc]) @ Cocc.T
    res.engine.set_charges(mol.Z)
    dS, dT, dV = res.engine.oei_deriv(1)
    g = 2.0 * torch.einsum("xij,ij->x", dT + dV, D) - 2.0 * torch.einsum("xij,ij->x", dS, W)
    g = (g + res.engine.grad_adjoint(D, 2.0, -1.0)).cpu().numpy()
    g += nuclear_repulsion(mol.Z, mol.coords, deriv=True)[1]
    return res.energy, g
