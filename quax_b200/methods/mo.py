"""AO -> MO transforms of the two-electron integrals on the GPU, and the RHF-MP2
energy as their first consumer.

Mirrors quax/methods/energy_utils.py:47-72 (tei_transformation,
partial_tei_transformation: four successive contractions of one AO index with a
coefficient block each) and the closed-shell MP2 of quax/methods/mp2.py:9-60.
Each quarter transform is one dense FP64 matrix product (cuBLAS DGEMM, FP64
tensor cores on B200) over the device-resident tensor; the reference runs them as
jnp.tensordot on the host.
"""
from __future__ import annotations

import torch


def _quarter(G: torch.Tensor, C: torch.Tensor) -> torch.Tensor:
    """tensordot(C, G, axes=[(0,), (3,)]) of the reference: contracts G's last index
    with C's first and puts the new index first (the next transform then sees the
    following index last)."""
    n = G.shape[-1]
    out = (G.reshape(-1, n) @ C).reshape(*G.shape[:-1], C.shape[1])
    return torch.movedim(out, -1, 0).contiguous()


def partial_tei_transformation(G: torch.Tensor, Ci, Cj, Ck, Cl) -> torch.Tensor:
    """(PQ|RS) = sum_pqrs G_pqrs Ci_pP Cj_qQ Ck_rR Cl_sS, four quarter transforms."""
    G = _quarter(G, Cl)
    G = _quarter(G, Ck)
    G = _quarter(G, Cj)
    return _quarter(G, Ci)


def tei_transformation(G: torch.Tensor, C) -> torch.Tensor:
    return partial_tei_transformation(G, C, C, C, C)


def rmp2_correlation(G_ao: torch.Tensor, C: torch.Tensor, eps: torch.Tensor, ndocc: int, ncore: int = 0) -> float:
    """Closed-shell MP2 correlation energy from the AO integrals (mp2.py:20-60):
    E = sum_ijab (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b)."""
    Co, Cv = C[:, ncore:ndocc], C[:, ndocc:]
    g = partial_tei_transformation(G_ao, Co, Cv, Co, Cv)  # (i a | j b)
    eo, ev = eps[ncore:ndocc], eps[ndocc:]
    denom = eo[:, None, None, None] - ev[None, :, None, None] + eo[None, None, :, None] - ev[None, None, None, :]
    return float(torch.sum(g * (2.0 * g - g.permute(0, 3, 2, 1)) / denom))
