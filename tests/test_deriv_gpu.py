"""GPU parity of the ERI derivative paths against the CPU oracle (through the C ABI).

Tolerances: derivative integrals 1e-11 absolute (the values reach O(10) for tight
primitives, so this is ~1e-12 relative); contracted gradients 1e-9 absolute.
"""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu
ATOL_D = 1e-11
ATOL_G = 1e-9


def _engine(basis, tol):
    from quax_b200.integrals.engine import EriEngine

    return EriEngine(basis, tol)


def small_synthetic(seed, natom=3, kmax=3):
    spec = SyntheticSpec(natom=natom, box=5.0, min_sep=1.2, kmax=kmax, exp_lo=0.1, exp_hi=50.0)
    return synthetic_molecule(spec, seed)[1]


def density(n, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, max(1, n // 4)))
    return C @ C.T


def test_h2o_deriv_core(oracle_lib):
    b = build_basis(h2o_config1(), "sto-3g")
    eng = _engine(b, 1e-14)
    d = eng.eri_deriv_core().cpu().numpy()
    ref = oracle_lib.eri_deriv1(oracle_lib.OracleBasis(b), 1e-14)
    assert d.shape == (9, 7, 7, 7, 7)
    assert np.abs(d - ref).max() < ATOL_D


@pytest.mark.parametrize("seed", [0, 4])
def test_synthetic_deriv_core(oracle_lib, seed):
    b = small_synthetic(seed)
    eng = _engine(b, 1e-12)
    d = eng.eri_deriv_core().cpu().numpy()
    ref = oracle_lib.eri_deriv1(oracle_lib.OracleBasis(b), 1e-12)
    assert np.abs(d - ref).max() < ATOL_D * max(1.0, np.abs(ref).max())


def test_deriv_slice(oracle_lib):
    b = small_synthetic(1)
    eng = _engine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    for nu in (0, 4, 3 * b.natom - 1):
        dv = np.zeros(3 * b.natom, dtype=int)
        dv[nu] = 1
        s = eng.eri_deriv(dv).cpu().numpy()
        ref = oracle_lib.eri_deriv1(ob, 1e-12, deriv_idx=nu)
        assert np.abs(s - ref).max() < ATOL_D * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("seed", [0, 2])
def test_grad_adjoint_matches_oracle_and_plain(oracle_lib, seed):
    b = small_synthetic(seed, natom=4)
    eng = _engine(b, 1e-12)
    n = eng.nbf
    D = density(n, seed)
    g = eng.grad_adjoint(torch.from_numpy(D), 1.0, -0.5).cpu().numpy()
    ref = oracle_lib.grad_contract(oracle_lib.OracleBasis(b), 1e-12, D, 1.0, -0.5)
    assert np.abs(g - ref).max() < ATOL_G
    # plain path: materialise the derivative tensor and contract with Gamma
    dG = eng.eri_deriv_core()
    Dt = torch.from_numpy(D).cuda()
    Gam = torch.einsum("ij,kl->ijkl", Dt, Dt) - 0.5 * torch.einsum("ik,jl->ijkl", Dt, Dt)
    gp = torch.einsum("xijkl,ijkl->x", dG, Gam).cpu().numpy()
    assert np.abs(g - gp).max() < ATOL_G
    # translational invariance of the contracted gradient
    assert np.abs(g.reshape(-1, 3).sum(axis=0)).max() < 1e-9


def sp_synthetic(seed, natom=3, kmax=3):
    spec = SyntheticSpec(natom=natom, box=5.0, min_sep=1.2, kmax=kmax, exp_lo=0.1, exp_hi=50.0,
                         heavy_ls=(0, 0, 1, 1), h_ls=(0, 1))
    return synthetic_molecule(spec, seed)[1]


def test_h2o_deriv2_core(oracle_lib):
    b = build_basis(h2o_config1(), "sto-3g")
    eng = _engine(b, 1e-14)
    d = eng.eri_deriv_core(2).cpu().numpy()
    ref = oracle_lib.eri_deriv2(oracle_lib.OracleBasis(b), 1e-14)
    assert d.shape == (45, 7, 7, 7, 7)
    assert np.abs(d - ref).max() < ATOL_D * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("seed", [0, 3])
def test_synthetic_deriv2_core(oracle_lib, seed):
    b = sp_synthetic(seed)
    eng = _engine(b, 1e-12)
    d = eng.eri_deriv_core(2).cpu().numpy()
    ref = oracle_lib.eri_deriv2(oracle_lib.OracleBasis(b), 1e-12)
    assert np.abs(d - ref).max() < ATOL_D * max(1.0, np.abs(ref).max())
    # symmetry of each slice under the 8 permutations of (ij|kl)
    assert np.abs(d - d.transpose(0, 2, 1, 3, 4)).max() < 1e-13 * max(1.0, np.abs(d).max())
    assert np.abs(d - d.transpose(0, 3, 4, 1, 2)).max() < 1e-13 * max(1.0, np.abs(d).max())


def test_deriv2_slices(oracle_lib):
    from quax_b200.utils import get_deriv_vec_idx

    b = sp_synthetic(5, natom=4)
    eng = _engine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    M = 3 * b.natom
    full = eng.eri_deriv_core(2).cpu().numpy()
    for nu1, nu2 in ((0, 0), (0, 1), (2, 7), (4, M - 1), (M - 1, M - 1)):
        dv = np.zeros(M, dtype=int)
        dv[nu1] += 1
        dv[nu2] += 1
        s = eng.eri_deriv(dv).cpu().numpy()
        r = get_deriv_vec_idx(dv)
        ref = oracle_lib.eri_deriv2(ob, 1e-12, pair_idx=r)
        assert np.abs(s - ref).max() < ATOL_D * max(1.0, np.abs(ref).max())
        assert np.abs(s - full[r]).max() < 1e-13 * max(1.0, np.abs(ref).max())


def test_deriv2_translational_invariance():
    # sum over the atoms of one Cartesian direction of d^2/dnu1 dnu2 vanishes
    b = sp_synthetic(2)
    eng = _engine(b, 1e-12)
    M = 3 * b.natom
    d = eng.eri_deriv_core(2).cpu().numpy()
    H = np.zeros((M, M) + d.shape[1:])
    r = 0
    for a in range(M):
        for c in range(a, M):
            H[a, c] = H[c, a] = d[r]
            r += 1
    for x in range(3):
        s = H[x::3].sum(axis=0)
        assert np.abs(s).max() < 1e-10 * max(1.0, np.abs(d).max())


def test_deriv_errors():
    b = small_synthetic(0)  # carries d shells
    eng = _engine(b, 1e-12)
    with pytest.raises(NotImplementedError):
        eng.eri_deriv_core(order=5)
    with pytest.raises(NotImplementedError):
        eng.eri_deriv_core(order=0)
    dv = np.zeros(3 * b.natom, dtype=int)
    dv[0] = 5
    with pytest.raises(NotImplementedError):
        eng.eri_deriv(dv)
    dv[0] = -1
    with pytest.raises(ValueError):
        eng.eri_deriv(dv)
    with pytest.raises(NotImplementedError):
        eng.eri_deriv(np.zeros(3 * b.natom, dtype=int))  # order 0
    with pytest.raises(ValueError):
        eng.eri_deriv(np.zeros(5, dtype=int))


def _unpack_hessian_slices(d2, M):
    """(M(M+1)/2, ...) unique nu1 <= nu2 slices -> (M, M, ...) symmetric."""
    H = np.zeros((M, M) + d2.shape[1:])
    r = 0
    for a in range(M):
        for c in range(a, M):
            H[a, c] = H[c, a] = d2[r]
            r += 1
    return H


@pytest.mark.parametrize("seed", [0, 3])
def test_grad_adjoint_jvp(seed):
    """Hessian-vector product of sum Gamma G (Gamma fixed) against (a) the order-2
    tensor contracted with Gamma and v, and (b) central differences of the adjoint
    gradient along v (h = 1e-4 bohr; tolerance 1e-6 relative)."""
    b = sp_synthetic(seed)
    eng = _engine(b, 1e-12)
    n, M = eng.nbf, 3 * b.natom
    D = density(n, seed)
    Dt = torch.from_numpy(D).cuda()
    rng = np.random.default_rng(seed)
    v = rng.normal(size=M)
    hv = eng.grad_adjoint_jvp(Dt, v, 1.0, -0.5).cpu().numpy()
    # (a) dense order-2 tensor
    H = _unpack_hessian_slices(eng.eri_deriv_core(2).cpu().numpy(), M)
    Gam = np.einsum("ij,kl->ijkl", D, D) - 0.5 * np.einsum("ik,jl->ijkl", D, D)
    HG = np.einsum("abijkl,ijkl->ab", H, Gam)
    assert np.abs(hv - HG @ v).max() < 1e-9 * max(1.0, np.abs(HG).max())
    # (b) central differences of the adjoint gradient
    h = 1e-4
    X = b.atom_coords().reshape(-1)
    gp = _engine(b.with_coords((X + h * v).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5).cpu().numpy()
    gm = _engine(b.with_coords((X - h * v).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5).cpu().numpy()
    fd = (gp - gm) / (2 * h)
    assert np.abs(hv - fd).max() < 1e-6 * max(1.0, np.abs(fd).max())
    # a unit vector gives one Hessian column
    e0 = np.zeros(M)
    e0[1] = 1.0
    col = eng.grad_adjoint_jvp(Dt, e0, 1.0, -0.5).cpu().numpy()
    assert np.abs(col - HG[:, 1]).max() < 1e-9 * max(1.0, np.abs(HG).max())


def test_grad_adjoint_jvp_errors():
    eng = _engine(small_synthetic(0), 1e-12)
    D = torch.eye(eng.nbf, dtype=torch.float64).cuda()
    assert np.abs(eng.grad_adjoint_jvp(D, np.zeros(3 * eng.natom)).cpu().numpy()).max() == 0.0
    with pytest.raises(ValueError):
        eng.grad_adjoint_jvp(D, np.zeros(5))
