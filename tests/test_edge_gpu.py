"""Edge cases of the ERI path against the oracle (GPU): a single shell on one atom
(one quartet per class), atoms 30 bohr apart (Boys arguments far beyond the
tabulated range, asymptotic branch), exponents from 0.01 to 1e5 (T near 0 and
huge prefactors), a loose threshold that screens most quartets, and the unique
quartet counts.  Tolerance 1e-12 absolute (relative for values above 1)."""
import numpy as np
import pytest

from quax_b200.basis import Basis, Shell, SyntheticSpec, synthetic_molecule

pytestmark = pytest.mark.gpu


def _check(oracle_lib, b, tol):
    from quax_b200.integrals.engine import EriEngine

    eng = EriEngine(b, tol)
    ob = oracle_lib.OracleBasis(b)
    G = eng.eri().cpu().numpy()
    ref = oracle_lib.compute_2e_int(ob, tol)
    assert np.abs(G - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    assert eng.unique_quartets() == oracle_lib.count_unique(ob, tol)
    eng.close()
    return eng


@pytest.mark.parametrize("l", [0, 1, 2])
def test_single_shell(oracle_lib, l):
    b = Basis([Shell(l, np.array([1.7, 0.3]), np.array([0.4, 0.7]), np.zeros(3), 0)], 1, False, "edge")
    _check(oracle_lib, b, 1e-14)


def test_far_apart_and_extreme_exponents(oracle_lib):
    shells = [
        Shell(0, np.array([1.0e5, 3.0e3, 90.0]), np.array([0.2, 0.5, 0.6]), np.zeros(3), 0),
        Shell(1, np.array([0.01]), np.array([1.0]), np.zeros(3), 0),
        Shell(2, np.array([4.0, 0.05]), np.array([0.5, 0.5]), np.array([0.0, 0.0, 30.0]), 1),
        Shell(1, np.array([2.5e4, 7.0]), np.array([0.3, 0.8]), np.array([0.0, 0.0, 30.0]), 1),
    ]
    _check(oracle_lib, Basis(shells, 2, False, "edge"), 1e-14)


def test_loose_threshold_screens_most_quartets(oracle_lib):
    from quax_b200.basis import SyntheticSpec, synthetic_molecule

    spec = SyntheticSpec(natom=4, box=12.0, min_sep=3.0, kmax=3, exp_lo=0.5, exp_hi=50.0)
    b = synthetic_molecule(spec, 2)[1]
    loose = oracle_lib.count_unique(oracle_lib.OracleBasis(b), 1e-4)
    tight = oracle_lib.count_unique(oracle_lib.OracleBasis(b), 1e-14)
    assert loose < tight
    _check(oracle_lib, b, 1e-4)


def test_bounded_wait_timeout_reports_device_error(oracle_lib):
    """Failure detection without a GPU fault: with a wait limit of 0 the split-mode
    kernels' bounded waits on their staging copies run out, the kernels report it
    through the error word (after letting the copies land) and return, and the
    host call raises; with the limit restored the same handle computes the oracle's
    tensor again (the error word was cleared)."""
    from quax_b200.integrals import _lib
    from quax_b200.integrals.engine import EriEngine

    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=4, exp_lo=0.1, exp_hi=50.0, charges=(6, 8))
    b = synthetic_molecule(spec, 3)[1]
    eng = EriEngine(b, 1e-12)
    forced = 0
    for c in eng.class_info():
        if c["nq"]:
            try:
                eng.set_engine(c["cls"], plain="wsplit")
                forced += 1
            except NotImplementedError:
                pass
    assert forced > 0
    eng.set_wait_limit(0)
    with pytest.raises(_lib.QuaxError, match="error word"):
        eng.eri_host()
    eng.set_wait_limit(1 << 22)
    G = eng.eri_host().reshape(eng.nbf, eng.nbf, eng.nbf, eng.nbf)
    ref = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)
    assert np.abs(G - ref).max() < 1e-12


def test_release_scratch_then_gradient_again():
    """qx_release_scratch frees the cached derivative accumulators; the next
    gradient allocates them again and gives the same result (1e-12)."""
    import torch

    from quax_b200.integrals.engine import EriEngine

    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=4, exp_lo=0.1, exp_hi=50.0)
    b = synthetic_molecule(spec, 3)[1]
    eng = EriEngine(b, 1e-12)
    n = eng.nbf
    C = np.random.default_rng(0).normal(0.0, 1.0 / np.sqrt(n), size=(n, n // 4))
    D = torch.from_numpy(C @ C.T).cuda()
    g1 = eng.grad_adjoint(D).cpu().numpy()
    eng.release_scratch()
    eng.release_scratch()  # twice: nothing left to free
    g2 = eng.grad_adjoint(D).cpu().numpy()
    assert np.abs(g1 - g2).max() < 1e-12
    eng.close()
