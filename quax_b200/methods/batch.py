"""Batched RHF: many molecules or geometries, J/K of the whole batch in one CUDA graph.

The reference runs one molecule per process through JAX (quax/methods/
hartree_fock.py:8-119).  Here a batch of molecules of different sizes shares the
GPU: every molecule keeps its own integral handle (its quartets sorted by class),
and the J/K builds of all molecules for one SCF iteration are captured once into a
CUDA graph -- each molecule's class launches on one of several side streams, so
the graph runs molecules side by side -- and replayed every iteration with the
densities updated in place.  After the SCF, the analytic gradient of every
molecule comes from the GPU one-electron derivative integrals and the adjoint
two-electron kernel.

The SCF is the reference's (Cholesky orthogonalisation, D = C_occ C_occ^T,
F = H + 2J - K, E = sum (F + H) D + E_nuc) with Pulay DIIS, run for a fixed
number of iterations as the batched workload specifies.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ..basis import Basis, Molecule
from ..integrals.engine import EriEngine
from ..oei import nuclear_repulsion


@dataclass
class _Mol:
    mol: Molecule
    basis: Basis
    eng: EriEngine
    A: torch.Tensor
    H: torch.Tensor
    S: torch.Tensor
    Enuc: float
    ndocc: int
    D: torch.Tensor
    J: torch.Tensor
    K: torch.Tensor
    dD: torch.Tensor = None  # incremental builds: density change and its J/K
    Jd: torch.Tensor = None
    Kd: torch.Tensor = None
    Dold: torch.Tensor = None
    F: torch.Tensor = None
    C: torch.Tensor = None
    eps: torch.Tensor = None
    E: float = 0.0
    focks: list = field(default_factory=list)
    errs: list = field(default_factory=list)


class BatchedRHF:
    def __init__(self, molecules, bases, ints_tol: float = 1.0e-12, streams: int = 8, autotune: bool = False,
                 incremental: float = 0.0, rebuild_every: int = 8):
        """incremental > 0: after the first iteration, J and K are updated from the
        density change with density screening at that threshold (qx_jk_screened),
        and rebuilt in full every `rebuild_every` iterations."""
        if len(molecules) != len(bases):
            raise ValueError("one basis per molecule")
        self.dev = torch.device("cuda")
        self.mols = []
        t0 = time.perf_counter()
        for mol, b in zip(molecules, bases):
            eng = EriEngine(b, ints_tol, device=self.dev)
            eng.set_charges(mol.Z)
            if autotune:
                eng.autotune()
            S, T, V = eng.oei()
            A = torch.linalg.inv(torch.linalg.cholesky(S)).T
            n = eng.nbf
            z = lambda: torch.zeros((n, n), dtype=torch.float64, device=self.dev)
            self.mols.append(_Mol(mol, b, eng, A, T + V, S, nuclear_repulsion(mol.Z, mol.coords),
                                  mol.nelectron // 2, z(), z(), z(), z(), z(), z(), z()))
        torch.cuda.synchronize()
        self.setup_s = time.perf_counter() - t0
        self.side = [torch.cuda.Stream(device=self.dev) for _ in range(streams)]
        self.graph = None
        self.graph_inc = None
        self.incremental = incremental
        self.rebuild_every = rebuild_every

    # -- J/K of the whole batch ---------------------------------------------------
    def _jk_all(self, inc: bool = False):
        cur = torch.cuda.current_stream()
        used = self.side[: min(len(self.side), len(self.mols))]
        for s in used:  # fork every used side stream from the current one (joins the capture)
            s.wait_stream(cur)
        for k, m in enumerate(self.mols):
            if inc:
                m.eng.jk(m.dD, m.Jd, m.Kd, stream=used[k % len(used)], screen=self.incremental)
            else:
                m.eng.jk(m.D, m.J, m.K, stream=used[k % len(used)])
        for s in used:
            cur.wait_stream(s)

    def capture(self):
        """Record the batch's J/K builds into CUDA graphs (after a warm-up run that
        makes every lazy allocation of the handles): the full build from D, and with
        incremental builds the screened build from the density change."""
        for inc in ((False, True) if self.incremental > 0 else (False,)):
            self._jk_all(inc)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._jk_all(inc)
            torch.cuda.synchronize()
            if inc:
                self.graph_inc = g
            else:
                self.graph = g

    def jk(self, inc: bool = False):
        if inc:
            for m in self.mols:
                torch.sub(m.D, m.Dold, out=m.dD)
            if self.graph_inc is not None:
                self.graph_inc.replay()
            else:
                self._jk_all(True)
            for m in self.mols:
                m.J += m.Jd
                m.K += m.Kd
        elif self.graph is not None:
            self.graph.replay()
        else:
            self._jk_all()
        for m in self.mols:
            m.Dold.copy_(m.D)

    # -- SCF -------------------------------------------------------------------
    def _diag(self, m: _Mol, F: torch.Tensor):
        Fp = m.A.T @ F @ m.A
        eps, C2 = torch.linalg.eigh(Fp)
        m.eps, m.C = eps, m.A @ C2
        Cocc = m.C[:, : m.ndocc]
        m.D.copy_(Cocc @ Cocc.T)  # in place: the graph reads these buffers

    def scf(self, iterations: int = 20, use_graph: bool = True):
        for m in self.mols:
            self._diag(m, m.H)
        if use_graph and self.graph is None:
            self.capture()
        t_jk = 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for it in range(iterations):
            inc = self.incremental > 0 and it % self.rebuild_every != 0
            e0.record()
            self.jk(inc)
            e1.record()
            torch.cuda.synchronize()
            t_jk += e0.elapsed_time(e1) * 1e-3
            for m in self.mols:
                F = m.H + 2.0 * m.J - m.K
                m.E = float(torch.sum((F + m.H) * m.D)) + m.Enuc
                err = m.A.T @ (F @ m.D @ m.S - m.S @ m.D @ F) @ m.A
                m.focks.append(F)
                m.errs.append(err)
                if len(m.focks) > 8:
                    m.focks.pop(0)
                    m.errs.pop(0)
                if len(m.focks) >= 2:
                    q = len(m.focks)
                    B = torch.empty((q + 1, q + 1), dtype=F.dtype, device=self.dev)
                    B[-1, :] = -1.0
                    B[:, -1] = -1.0
                    B[-1, -1] = 0.0
                    for i in range(q):
                        for j in range(q):
                            B[i, j] = torch.sum(m.errs[i] * m.errs[j])
                    rhs = torch.zeros(q + 1, dtype=F.dtype, device=self.dev)
                    rhs[-1] = -1.0
                    c = torch.linalg.lstsq(B, rhs.unsqueeze(1)).solution.squeeze(1)
                    F = sum(c[i] * m.focks[i] for i in range(q))
                self._diag(m, F)
        # energies at the final densities
        self.jk()
        torch.cuda.synchronize()
        for m in self.mols:
            F = m.H + 2.0 * m.J - m.K
            m.E = float(torch.sum((F + m.H) * m.D)) + m.Enuc
            self._diag(m, F)
            Cocc = m.C[:, : m.ndocc]
            m.D.copy_(Cocc @ Cocc.T)
        return [m.E for m in self.mols], t_jk

    # -- gradients ---------------------------------------------------------------
    def gradients(self):
        """Analytic RHF gradient of every molecule at its current orbitals."""
        out = []
        for m in self.mols:
            Cocc = m.C[:, : m.ndocc]
            D = Cocc @ Cocc.T
            W = Cocc @ torch.diag(m.eps[: m.ndocc]) @ Cocc.T
            dS, dT, dV = m.eng.oei_deriv(1)
            g = 2.0 * torch.einsum("xij,ij->x", dT + dV, D) - 2.0 * torch.einsum("xij,ij->x", dS, W)
            g = g + m.eng.grad_adjoint(D, 2.0, -1.0)
            out.append(g.cpu().numpy() + nuclear_repulsion(m.mol.Z, m.mol.coords, deriv=True)[1])
            del dS, dT, dV
            m.eng.release_scratch()  # one molecule's derivative accumulators at a time
        return out

    def close(self):
        self.graph = None
        self.graph_inc = None
        for m in self.mols:
            m.eng.close()


def displaced_geometries(mol: Molecule, count: int, sigma: float, seed: int = 0):
    """Gaussian-displaced copies of a molecule (sigma in bohr)."""
    rng = np.random.default_rng(seed)
    return [Molecule(mol.Z.copy(), mol.coords + rng.normal(0.0, sigma, size=mol.coords.shape), mol.charge)
            for _ in range(count)]
