"""AO -> MO transforms on the GPU against a host einsum, and the RHF-MP2 correlation
energy of H2O/STO-3G against the same formula evaluated with numpy (1e-12)."""
import numpy as np
import pytest
import torch

from quax_b200.basis import build_basis, h2o_config1

pytestmark = pytest.mark.gpu


def test_partial_transform_and_mp2():
    from quax_b200.methods.hartree_fock import restricted_hartree_fock
    from quax_b200.methods.mo import partial_tei_transformation, rmp2_correlation

    mol = h2o_config1()
    res = restricted_hartree_fock(mol, build_basis(mol, "sto-3g"), conv=1e-11)
    G = res.engine.eri()
    C = res.C
    rng = np.random.default_rng(0)
    Cs = [torch.from_numpy(rng.normal(size=(7, k))).cuda() for k in (2, 3, 4, 5)]
    out = partial_tei_transformation(G, *Cs).cpu().numpy()
    ref = np.einsum("pqrs,pP,qQ,rR,sS->PQRS", G.cpu().numpy(), *[c.cpu().numpy() for c in Cs], optimize=True)
    assert np.abs(out - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    ndocc = mol.nelectron // 2
    e = rmp2_correlation(G, C, res.eps, ndocc)
    Gh, Ch, eh = G.cpu().numpy(), C.cpu().numpy(), res.eps.cpu().numpy()
    g = np.einsum("pqrs,pi,qa,rj,sb->iajb", Gh, Ch[:, :ndocc], Ch[:, ndocc:], Ch[:, :ndocc], Ch[:, ndocc:])
    eo, ev = eh[:ndocc], eh[ndocc:]
    d = eo[:, None, None, None] - ev[None, :, None, None] + eo[None, None, :, None] - ev[None, None, None, :]
    e_ref = np.sum(g * (2 * g - g.transpose(0, 3, 2, 1)) / d)
    assert abs(e - e_ref) < 1e-12 and -0.2 < e < 0.0
