"""Sharded handles on one GPU: the per-rank results of qx_set_shard sum to the
full ones (dense ERI, derivative tensor, J/K, adjoint gradient), and the ranks'
unique quartets partition the full list.  Each rank is a separate handle run one
after the other, so nothing waits on another rank (the all-reduce itself is
covered by the gloo tests on CPU).  Tolerances as in the other GPU tests."""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, synthetic_molecule

pytestmark = pytest.mark.gpu


def _basis(seed, natom=4):
    spec = SyntheticSpec(natom=natom, box=6.0, min_sep=1.2, kmax=4, exp_lo=0.1, exp_hi=80.0)
    return synthetic_molecule(spec, seed)[1]


@pytest.mark.parametrize("nranks", [2, 3])
def test_shards_sum_to_full(nranks):
    from quax_b200.integrals.engine import EriEngine

    b = _basis(1)
    full = EriEngine(b, 1e-12)
    n = full.nbf
    rng = np.random.default_rng(5)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, max(1, n // 4)))
    D = torch.from_numpy(C @ C.T).cuda()
    G = full.eri()
    dG = full.eri_deriv_core()
    J, K = full.jk(D)
    g = full.grad_adjoint(D)
    nq = full.unique_quartets()
    sG, sdG, sJ, sK, sg, snq = 0, 0, 0, 0, 0, 0
    for r in range(nranks):
        e = EriEngine(b, 1e-12)
        e.set_shard(r, nranks)
        e.autotune()  # engines re-chosen for the smaller lists
        sG = sG + e.eri()
        sdG = sdG + e.eri_deriv_core()
        Jr, Kr = e.jk(D)
        sJ, sK = sJ + Jr, sK + Kr
        sg = sg + e.grad_adjoint(D)
        snq += e.unique_quartets()
        assert 0 < e.unique_quartets() < nq
        e.close()
    assert snq == nq
    assert (sG - G).abs().max().item() < 1e-12
    # the ranks' autotuned engines may differ from the full handle's (the Rys engine
    # differentiates all four centres, the Obara-Saika engines take the fourth by
    # translational invariance): on same-atom (dd|dd) quartets with tight exponents
    # the invariance sum loses up to 6.5e-11 (quartet (20,5|20,5) of this molecule
    # against a 40-digit evaluation; the direct derivative is within 2e-16), so
    # cross-engine derivative tensors agree to 1e-10
    assert (sdG - dG).abs().max().item() < 1e-10 * max(1.0, dG.abs().max().item())
    assert (sJ - J).abs().max().item() < 1e-11
    assert (sK - K).abs().max().item() < 1e-11
    assert (sg - g).abs().max().item() < 1e-9


def test_shard_restore_and_errors():
    from quax_b200.integrals.engine import EriEngine

    b = _basis(2, natom=3)
    e = EriEngine(b, 1e-12)
    nq = e.unique_quartets()
    out = torch.empty(e.unique_size(), dtype=torch.float64, device="cuda")
    e.eri_unique(out)
    e.set_shard(1, 2)
    assert e.unique_quartets() < nq
    e.set_shard(0, 1)
    assert e.unique_quartets() == nq
    out2 = torch.empty(e.unique_size(), dtype=torch.float64, device="cuda")
    e.eri_unique(out2)
    assert (out2 - out).abs().max().item() < 1e-13
    for bad in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(ValueError):
            e.set_shard(*bad)
