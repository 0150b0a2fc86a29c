"""Host one-electron integrals (consumed by the RHF driver) against finite differences
and basic identities; CPU only."""
import numpy as np

from quax_b200.basis import build_basis, h2o_config1
from quax_b200.oei import boys_host, nuclear_repulsion, one_electron


def test_overlap_diagonal_and_symmetry():
    mol = h2o_config1()
    S, T, V = one_electron(build_basis(mol, "sto-3g"), mol.Z, mol.coords)
    assert np.allclose(np.diag(S)[[0, 1, 2, 5, 6]], 1.0, atol=1e-12)  # s and x^1 components
    for M in (S, T, V):
        assert np.array_equal(M, M.T)


def test_derivatives_against_finite_differences():
    mol = h2o_config1()
    b = build_basis(mol, "sto-3g")
    S, T, V, dS, dT, dV = one_electron(b, mol.Z, mol.coords, deriv=True)
    h = 1e-4
    for nu in (0, 2, 4, 7):
        c = mol.coords.copy()
        c.flat[nu] += h
        Sp, Tp, Vp = one_electron(b.with_coords(c), mol.Z, c)
        c.flat[nu] -= 2 * h
        Sm, Tm, Vm = one_electron(b.with_coords(c), mol.Z, c)
        for d, p, m in ((dS, Sp, Sm), (dT, Tp, Tm), (dV, Vp, Vm)):
            assert np.abs(d[nu] - (p - m) / (2 * h)).max() < 1e-7


def test_nuclear_repulsion_gradient():
    mol = h2o_config1()
    E, g = nuclear_repulsion(mol.Z, mol.coords, deriv=True)
    h = 1e-5
    for nu in range(9):
        c = mol.coords.copy()
        c.flat[nu] += h
        ep = nuclear_repulsion(mol.Z, c)
        c.flat[nu] -= 2 * h
        em = nuclear_repulsion(mol.Z, c)
        assert abs(g[nu] - (ep - em) / (2 * h)) < 1e-7


def test_boys_host_limits():
    assert np.allclose(boys_host(4, 0.0), 1.0 / np.array([1, 3, 5, 7, 9]))
    T = 60.0
    assert abs(boys_host(0, T)[0] - 0.5 * np.sqrt(np.pi / T)) < 1e-15
