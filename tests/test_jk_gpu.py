"""Direct J/K against contractions of the dense ERI tensor (GPU).

The reference builds J = jk_build(G, D) and K = jk_build(G.transpose(0,2,1,3), D)
from the dense tensor (quax/methods/hartree_fock.py:26-28,79-80); the direct build
must give the same matrices.  Tolerance 1e-11 absolute (sums of ~n^2 integrals of
size <= 1e-12 error each)."""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["h2o", "syn0", "syn3"])
def test_jk_matches_dense_contraction(oracle_lib, which):
    from quax_b200.integrals.engine import EriEngine

    if which == "h2o":
        b = build_basis(h2o_config1(), "sto-3g")
    else:
        spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0)
        b = synthetic_molecule(spec, int(which[-1]))[1]
    eng = EriEngine(b, 1e-12)
    n = eng.nbf
    rng = np.random.default_rng(7)
    C = rng.normal(size=(n, max(1, n // 3)))
    D = C @ C.T / n
    J, K = eng.jk(torch.from_numpy(D))
    G = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)
    Jr = np.einsum("ijkl,kl->ij", G, D)
    Kr = np.einsum("ikjl,kl->ij", G, D)
    assert np.abs(J.cpu().numpy() - Jr).max() < 1e-11
    assert np.abs(K.cpu().numpy() - Kr).max() < 1e-11


def test_jk_screened():
    """qx_jk_screened: threshold 0 equals qx_jk; with a threshold, the skipped
    quartets' contributions are bounded by it times the number of contributions,
    and a density change (incremental build) skips quartets but still adds up."""
    from quax_b200.integrals.engine import EriEngine

    spec = SyntheticSpec(natom=4, box=7.0, min_sep=1.3, kmax=3, exp_lo=0.1, exp_hi=50.0)
    b = synthetic_molecule(spec, 5)[1]
    eng = EriEngine(b, 1e-12)
    n = eng.nbf
    rng = np.random.default_rng(3)
    C = rng.normal(size=(n, max(1, n // 3)))
    D = torch.from_numpy(C @ C.T / n).cuda()
    J, K = eng.jk(D)
    J0, K0 = eng.jk(D, screen=0.0)
    Js, Ks = eng.jk(D, screen=1e-300)  # screening on, nothing below the threshold
    assert (Js - J).abs().max().item() < 1e-13 and (Ks - K).abs().max().item() < 1e-13
    Jt, Kt = eng.jk(D, screen=1e-11)
    assert (Jt - J).abs().max().item() < 1e-8 and (Kt - K).abs().max().item() < 1e-8
    # incremental: J(D + dD) = J(D) + J(dD), with dD small and screened
    dD = 1e-6 * torch.from_numpy(rng.normal(size=(n, n))).cuda()
    dD = dD + dD.T
    J2, K2 = eng.jk(D + dD)
    Jd, Kd = eng.jk(dD, screen=1e-12)
    assert (J + Jd - J2).abs().max().item() < 1e-9 and (K + Kd - K2).abs().max().item() < 1e-9
