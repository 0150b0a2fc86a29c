"""Mixed precision (qx_set_precision): quartets with Schwarz bound below a
threshold run their recurrences in FP32, everything else FP64.

Every result is compared with the all-FP64 GPU run of the same handle, and the
error is bounded in terms of the threshold: in the classes that may run FP32
(HRR with at most two transfer steps) the FP32 recurrences lose up to ~2e-3 of
the integral's magnitude, itself below the quartet's bound, so the tests allow
5e-3 x bound per integral, and the J/K and gradient errors that follow from it.  With the threshold at 0 the
results must be the FP64 ones."""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, synthetic_molecule

pytestmark = pytest.mark.gpu


def _basis(seed):
    spec = SyntheticSpec(natom=4, box=7.0, min_sep=1.4, kmax=4, exp_lo=0.1, exp_hi=200.0)
    return synthetic_molecule(spec, seed)[1]


@pytest.mark.parametrize("bound", [1e-8, 1e-6, 1e-4])
def test_mixed_against_fp64(bound):
    from quax_b200.integrals.engine import EriEngine

    b = _basis(1)
    ref = EriEngine(b, 1e-12)
    n = ref.nbf
    rng = np.random.default_rng(2)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, max(1, n // 4)))
    D = torch.from_numpy(C @ C.T).cuda()
    G = ref.eri()
    J, K = ref.jk(D)
    g = ref.grad_adjoint(D)
    e = EriEngine(b, 1e-12)
    e.set_precision(bound)
    split = e.precision_split()
    assert sum(v[0] for v in split.values()) < sum(v[1] for v in split.values())  # some quartets run FP32
    G2 = e.eri()
    J2, K2 = e.jk(D)
    g2 = e.grad_adjoint(D)
    dG = (G2 - G).abs().max().item()
    assert dG <= 5e-3 * bound
    assert (J2 - J).abs().max().item() <= 5e-3 * bound * n * n * D.abs().max().item()
    assert (g2 - g).abs().max().item() <= 1e3 * 5e-3 * bound
    if bound <= 1e-8:  # the 1e-8 Eh/bohr gradient budget holds at this threshold
        assert (g2 - g).abs().max().item() <= 1e-8
    # back to FP64: identical results up to summation order
    e.set_precision(0.0)
    assert all(v[0] == v[1] for v in e.precision_split().values())
    assert (e.eri() - G).abs().max().item() < 1e-13


def test_mixed_unique_layout_and_errors():
    from quax_b200.integrals.engine import EriEngine

    b = _basis(2)
    e = EriEngine(b, 1e-12)
    nq = e.unique_quartets()
    e.set_precision(1e-6)
    assert e.unique_quartets() == nq
    out = torch.empty(e.unique_size(), dtype=torch.float64, device="cuda")
    e.eri_unique(out)
    assert torch.isfinite(out).all()
    with pytest.raises(ValueError):
        e.set_precision(float("nan"))
