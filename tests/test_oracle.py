"""CPU checks that pin the FP64 oracle (test infrastructure for the GPU parity tests).

The reference's integral values come from Libint, which cannot be built here, and
the reference stores no golden integral vectors; the oracle is pinned instead by
  * published textbook values: Szabo & Ostlund, Modern Quantum Chemistry, H2 in
    STO-3G at R = 1.4 bohr (4 printed digits);
  * a closed form for (ss|ss) of single primitives;
  * the Boys function against mpmath's incomplete gamma function;
  * an independent McMurchie-Davidson implementation (oracle/md_check.py);
  * central finite differences of the oracle's own integrals;
  * permutational symmetry and translational invariance.
"""
import math

import numpy as np
import pytest

from oracle import md_check
from quax_b200.basis import Basis, Molecule, Shell, build_basis, h2o_config1


def test_szabo_ostlund_h2(oracle_lib):
    mol = Molecule(np.array([1, 1]), np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]]))
    G = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(build_basis(mol, "sto-3g")), 1e-14)
    assert round(G[0, 0, 0, 0], 4) == 0.7746
    assert round(G[0, 0, 1, 1], 4) == 0.5697
    assert round(G[1, 0, 0, 0], 4) == 0.4441
    assert round(G[1, 0, 1, 0], 4) == 0.2970


def test_closed_form_ssss(oracle_lib):
    a, b, c, d = 1.3, 0.7, 2.1, 0.4
    A, B, C, D = (np.array(v, float) for v in ([0, 0, 0], [0.5, 0, 0.2], [0, 1.1, 0], [0.3, 0.3, 0.9]))
    sh = [Shell(0, np.array([x]), np.array([1.0]), P, i) for i, (x, P) in enumerate(zip((a, b, c, d), (A, B, C, D)))]
    v = oracle_lib.shell_quartet(oracle_lib.OracleBasis(Basis(sh, 4)), 0, 1, 2, 3)[0, 0, 0, 0]
    p, q = a + b, c + d
    P = (a * A + b * B) / p
    Q = (c * C + d * D) / q
    T = p * q / (p + q) * np.sum((P - Q) ** 2)
    F0 = 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
    N = [(2 * x / math.pi) ** 0.75 for x in (a, b, c, d)]
    ref = (np.prod(N) * 2 * math.pi**2.5 / (p * q * math.sqrt(p + q)) * math.exp(-a * b / p * np.sum((A - B) ** 2))
           * math.exp(-c * d / q * np.sum((C - D) ** 2)) * F0)
    assert abs(v - ref) < 1e-15 * max(1.0, abs(ref))


@pytest.mark.parametrize("T", [0.0, 1e-10, 1e-3, 0.37, 2.5, 11.0, 29.99, 39.9, 44.99, 45.01, 80.0, 500.0])
def test_boys_against_mpmath(oracle_lib, T):
    f = oracle_lib.boys(16, T)
    ref = np.array([md_check._boys(m, T) for m in range(17)])
    assert np.max(np.abs(f / ref - 1.0)) < 5e-15


def _random_shells(seed, ls, k=2):
    rng = np.random.default_rng(seed)
    return [Shell(l, np.sort(np.exp(rng.uniform(-1.5, 2.0, k)))[::-1].copy(), rng.uniform(0.1, 1.0, k),
                  rng.uniform(-1.5, 1.5, 3), i) for i, l in enumerate(ls)]


@pytest.mark.parametrize("ls", [(0, 0, 0, 0), (1, 0, 1, 1), (2, 0, 1, 0), (2, 1, 2, 0), (1, 2, 0, 2), (2, 2, 1, 1)])
def test_mcmurchie_davidson_plain(oracle_lib, ls):
    sh = _random_shells(sum(ls) * 7 + ls[0], ls, k=2)
    o = oracle_lib.shell_quartet(oracle_lib.OracleBasis(Basis(sh, 4)), 0, 1, 2, 3)
    m = md_check.shell_quartet(sh)
    assert np.abs(o - m).max() < 1e-13 * max(1.0, np.abs(m).max())


@pytest.mark.parametrize("ls", [(0, 0, 0, 0), (1, 0, 0, 1), (2, 1, 0, 0)])
def test_mcmurchie_davidson_deriv(oracle_lib, ls):
    sh = _random_shells(31 + sum(ls), ls, k=1)
    o = oracle_lib.shell_quartet(oracle_lib.OracleBasis(Basis(sh, 4)), 0, 1, 2, 3, deriv=True)
    m = md_check.shell_quartet(sh, deriv=True)
    assert np.abs(o - m).max() < 1e-13 * max(1.0, np.abs(m).max())


def test_normalisation_xl_unit():
    for sh in _random_shells(5, (0, 1, 2), k=3):
        assert abs(md_check.overlap_xl(sh) - 1.0) < 1e-13


def test_dense_symmetry_h2o(oracle_lib):
    G = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(build_basis(h2o_config1(), "sto-3g")), 1e-14)
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1), (3, 2, 1, 0)]:
        assert np.abs(G - G.transpose(perm)).max() < 1e-15


def test_deriv_against_finite_differences(oracle_lib):
    """Five-point central differences (h = 1e-3 bohr, error O(h^4)) of the ERI tensor."""
    mol = h2o_config1()
    b = build_basis(mol, "sto-3g")
    d = oracle_lib.eri_deriv1(oracle_lib.OracleBasis(b), 1e-14)
    h = 1e-3
    for nu in (0, 4, 8):
        def G(shift):
            c = mol.coords.copy()
            c.flat[nu] += shift
            return oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b.with_coords(c)), 1e-14)
        fd = (G(-2 * h) - 8 * G(-h) + 8 * G(h) - G(2 * h)) / (12 * h)
        assert np.abs(d[nu] - fd).max() < 2e-9


def test_translational_invariance(oracle_lib):
    d = oracle_lib.eri_deriv1(oracle_lib.OracleBasis(build_basis(h2o_config1(), "sto-3g")), 1e-14)
    for x in range(3):
        assert np.abs(d[x::3].sum(axis=0)).max() < 1e-13


def test_gradient_oracle_matches_dense_contraction(oracle_lib):
    b = build_basis(h2o_config1(), "sto-3g")
    ob = oracle_lib.OracleBasis(b)
    rng = np.random.default_rng(1)
    C = rng.normal(size=(7, 3))
    D = C @ C.T
    Gam = np.einsum("ij,kl->ijkl", D, D) - 0.5 * np.einsum("ik,jl->ijkl", D, D)
    g_dense = np.einsum("xijkl,ijkl->x", oracle_lib.eri_deriv1(ob, 1e-14), Gam)
    g = oracle_lib.grad_contract(ob, 1e-14, D, 1.0, -0.5)
    assert np.abs(g - g_dense).max() < 1e-12


@pytest.mark.parametrize("ls", [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 0, 1)])
def test_second_derivatives_mcmurchie_davidson(oracle_lib, ls):
    sh = _random_shells(50 + sum(ls), ls, k=1)
    o = oracle_lib.shell_quartet_deriv2(oracle_lib.OracleBasis(Basis(sh, 4)), 0, 1, 2, 3)
    m = md_check.shell_quartet_deriv2(sh)
    assert np.abs(o - m).max() < 1e-12 * max(1.0, np.abs(m).max())


def test_second_derivative_tensor_against_finite_differences(oracle_lib):
    """d/dR_nu2 of the first-derivative slice nu1, five-point differences (h = 1e-3)."""
    mol = h2o_config1()
    b = build_basis(mol, "sto-3g")
    d2 = oracle_lib.eri_deriv2(oracle_lib.OracleBasis(b), 1e-14)
    assert d2.shape == (45, 7, 7, 7, 7)
    from quax_b200.utils import multiset_rank

    h = 1e-3
    for nu1, nu2 in [(0, 0), (0, 4), (2, 7), (5, 5)]:
        def d1(shift):
            c = mol.coords.copy()
            c.flat[nu2] += shift
            return oracle_lib.eri_deriv1(oracle_lib.OracleBasis(b.with_coords(c)), 1e-14, deriv_idx=nu1)
        fd = (d1(-2 * h) - 8 * d1(-h) + 8 * d1(h) - d1(2 * h)) / (12 * h)
        k = multiset_rank(sorted((nu1, nu2)), 9)
        assert np.abs(d2[k] - fd).max() < 5e-8
