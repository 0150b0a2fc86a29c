"""GPU parity of the ERI tensor against the CPU oracle (through the C ABI).

Tolerance: 1e-12 absolute per integral (the FP64 bar for the plain path).
"""
import numpy as np
import pytest

from quax_b200.basis import Basis, Molecule, Shell, SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu
ATOL = 1e-12


def _engine(basis, tol=1e-14):
    from quax_b200.integrals.engine import EriEngine

    return EriEngine(basis, tol)


def small_synthetic(seed, natom=3, kmax=4):
    spec = SyntheticSpec(natom=natom, box=5.0, min_sep=1.2, kmax=kmax, exp_lo=0.1, exp_hi=50.0)
    return synthetic_molecule(spec, seed)[1]


def test_h2o_sto3g_dense(oracle_lib):
    b = build_basis(h2o_config1(), "sto-3g")
    eng = _engine(b)
    G = eng.eri().cpu().numpy()
    ref = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-14)
    assert G.shape == (7, 7, 7, 7)
    assert np.abs(G - ref).max() < ATOL


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_synthetic_dense(oracle_lib, seed):
    b = small_synthetic(seed)
    eng = _engine(b, 1e-12)
    G = eng.eri().cpu().numpy()
    ref = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)
    assert np.abs(G - ref).max() < ATOL
    # 8-fold permutational symmetry (elements of one diagonal block are computed
    # separately, so images agree to rounding, not bitwise)
    assert np.abs(G - G.transpose(1, 0, 2, 3)).max() < 1e-14
    assert np.abs(G - G.transpose(2, 3, 0, 1)).max() < 1e-14


def test_schwarz_and_count(oracle_lib):
    b = small_synthetic(5, natom=4)
    eng = _engine(b, 1e-10)
    ob = oracle_lib.OracleBasis(b)
    K, kmax = eng.schwarz()
    Kr, kmaxr = oracle_lib.schwarz(ob)
    assert np.allclose(K, Kr, rtol=1e-12, atol=1e-300)
    assert eng.unique_quartets() == oracle_lib.count_unique(ob, 1e-10)


def test_host_buffer_matches_device():
    b = small_synthetic(3)
    eng = _engine(b)
    n = eng.nbf
    Gd = eng.eri().cpu().numpy()
    Gh = eng.eri_host().reshape(n, n, n, n)
    assert np.array_equal(Gd, Gh)


def test_unique_blocks(oracle_lib):
    """The compact unique layout holds each screened quartet's block once."""
    b = small_synthetic(7)
    eng = _engine(b, 1e-12)
    u = eng.eri_unique().cpu().numpy()
    assert u.size == eng.unique_size()
    G = eng.eri().cpu().numpy()
    # the sum of squares over unique blocks weighted by degeneracy equals the dense sum of squares
    assert np.isfinite(u).all()
    assert np.abs(u).max() == pytest.approx(np.abs(G).max(), rel=0, abs=0)
