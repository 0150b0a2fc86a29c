"""GPU parity of the Rys-quadrature engine (f shells, and derivatives of order >= 2
with d and f shells) against the CPU oracle, through the C ABI.

The oracle is an independent Obara-Saika / Head-Gordon-Pople restatement, so these
tests compare two different algorithms.  Tolerances: ERI 1e-12 absolute;
contracted gradients 1e-9 absolute scaled by max(1, max |value|); derivative
tensors with f shells 1e-9 absolute scaled likewise.  The last is looser than the
l <= 2 bar (1e-11) because the oracle itself is not reproducible to 1e-11 there:
the same (ff|df) quartet with a tight d shell (exponent 42.6) beside diffuse f
shells, evaluated by the oracle in two centre orders, differs by 2.9e-10 (quartet
(3,7|2,7) of f_synthetic(5, natom=2)); the Rys arithmetic matches the oracle's
original-order block to 1e-17 on that quartet.
"""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, synthetic_molecule

pytestmark = pytest.mark.gpu
ATOL = 1e-12
ATOL_DF = 1e-9  # derivative tensors with f shells
ATOL_D = 1e-11  # derivative tensors with d shells
ATOL_G = 1e-9
HIGH_ORDER_TOL = {3: 5e-8, 4: 1e-6}  # order-3/4 tensors: the oracle's error (see the tests)


def _engine(basis, tol):
    from quax_b200.integrals.engine import EriEngine

    return EriEngine(basis, tol)


def f_synthetic(seed, natom=3, heavy=(0, 1, 2), kmax=3):
    """Synthetic molecule whose heavy atoms carry s, p, d and an f shell (K 1-3,
    exponents in [0.2, 5], the large workload's f shells)."""
    spec = SyntheticSpec(natom=natom, box=5.0, min_sep=1.2, kmax=kmax, exp_lo=0.1, exp_hi=50.0, heavy_ls=heavy,
                         h_ls=(0, 1), f_shell=True)
    return synthetic_molecule(spec, seed)[1]


def density(n, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, max(1, n // 4)))
    return C @ C.T


def _has_f(b):
    return any(s.l == 3 for s in b.shells)


@pytest.mark.parametrize("seed", [0, 1])
def test_f_dense(oracle_lib, seed):
    b = f_synthetic(seed)
    assert _has_f(b)
    eng = _engine(b, 1e-12)
    G = eng.eri().cpu().numpy()
    ref = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)
    assert np.abs(G - ref).max() < ATOL


def test_f_schwarz_and_unique_blocks(oracle_lib):
    """Schwarz table, and every screened unique quartet of every class element by
    element against the oracle's block of the same canonical shell quartet."""
    b = f_synthetic(2)
    eng = _engine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    K, kmax = eng.schwarz()
    Kr, kmr = oracle_lib.schwarz(ob)
    assert np.abs(K - Kr).max() <= 1e-12 * max(1.0, kmr)
    nq = 0
    for cls, (sh, blk) in eng.unique_blocks().items():
        blk = blk.cpu().numpy()
        for q in range(sh.shape[0]):
            ref = oracle_lib.shell_quartet(ob, *[int(x) for x in sh[q]]).reshape(-1)
            assert np.abs(blk[q] - ref).max() < ATOL, (cls, q)
        nq += sh.shape[0]
    assert nq == eng.unique_quartets() == oracle_lib.count_unique(ob, 1e-12)


@pytest.mark.parametrize("all_rys", [False, True])
def test_f_jk(oracle_lib, all_rys):
    """Direct J/K with f shells (the Rys engine's block-contraction epilogue),
    with the default engines and with the Rys engine on every class, against the
    oracle's dense tensor contracted with D (1e-10)."""
    b = f_synthetic(3)
    eng = _engine(b, 1e-12)
    if all_rys:
        for c in eng.class_info():
            eng.set_engine(c["cls"], plain="rys")
    n = eng.nbf
    D = density(n, 3)
    J, Kx = eng.jk(torch.from_numpy(D).cuda())
    G = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)
    Jr = np.einsum("ijkl,kl->ij", G, D)
    Kr = np.einsum("ikjl,kl->ij", G, D)
    assert np.abs(J.cpu().numpy() - Jr).max() < 1e-10
    assert np.abs(Kx.cpu().numpy() - Kr).max() < 1e-10


@pytest.mark.parametrize("seed", [0, 5])
def test_f_deriv_core_and_slice(oracle_lib, seed):
    b = f_synthetic(seed, natom=2)
    eng = _engine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    d = eng.eri_deriv_core(1).cpu().numpy()
    ref = oracle_lib.eri_deriv1(ob, 1e-12)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(d - ref).max() < ATOL_DF * scale
    for nu in (0, 3 * b.natom - 1):
        dv = np.zeros(3 * b.natom, dtype=int)
        dv[nu] = 1
        s = eng.eri_deriv(dv).cpu().numpy()
        assert np.abs(s - ref[nu]).max() < ATOL_DF * scale


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("build", [None, 0, 1])
def test_f_grad_adjoint(oracle_lib, seed, build):
    """The adjoint gradient with the default engines, and with the Rys engine
    forced on every class with either table build (per-unit for small units, or
    level-parallel), against the oracle."""
    b = f_synthetic(seed)
    eng = _engine(b, 1e-12)
    if build is not None:
        for c in eng.class_info():
            eng.set_engine(c["cls"], deriv="rys", deriv_param=build)
    D = density(eng.nbf, seed)
    g = eng.grad_adjoint(torch.from_numpy(D).cuda(), 1.0, -0.5).cpu().numpy()
    gr = oracle_lib.grad_contract(oracle_lib.OracleBasis(b), 1e-12, D, 1.0, -0.5)
    assert np.abs(g - gr).max() < ATOL_G * max(1.0, np.abs(gr).max())


def _unpack_pairs(d2, M):
    H = np.zeros((M, M) + d2.shape[1:])
    r = 0
    for a in range(M):
        for c in range(a, M):
            H[a, c] = H[c, a] = d2[r]
            r += 1
    return H


@pytest.mark.parametrize("heavy", [(0, 2), (1,)])
def test_deriv2_with_d_and_f(oracle_lib, heavy):
    """Order-2 tensor (nuclear pairs nu1 <= nu2) with d and f shells, dense and one
    slice, against the oracle's order-2 tensor."""
    b = f_synthetic(4, natom=2, heavy=heavy, kmax=2)
    eng = _engine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    d2 = eng.eri_deriv_core(2).cpu().numpy()
    ref = oracle_lib.eri_deriv2(ob, 1e-12)
    scale = max(1.0, np.abs(ref).max())
    tol = ATOL_DF * scale  # every heavy atom carries an f shell
    assert np.abs(d2 - ref.reshape(d2.shape)).max() < tol
    M = 3 * b.natom
    dv = np.zeros(M, dtype=int)
    dv[1] += 1
    dv[M - 2] += 1
    s = eng.eri_deriv(dv).cpu().numpy()
    k = 1 * M - 0 + (M - 2 - 1)  # rank of (1, M-2): nu1*M - nu1(nu1-1)/2 + nu2 - nu1
    assert np.abs(s.reshape(-1) - ref.reshape(ref.shape[0], -1)[k]).max() < tol


def test_hessian_columns_with_d_and_f():
    """Hessian columns (unit directions: the quartets off the displaced atom are
    skipped, since every term is linear in the displacement) on a 3-atom molecule
    with d and f shells: the columns combined with v equal the product along v
    (where nothing is skipped) to 1e-10 relative, and one column matches central
    differences of the adjoint gradient (h = 1e-4 bohr, 1e-6 relative)."""
    b = f_synthetic(1, natom=3, kmax=2)
    eng = _engine(b, 1e-12)
    n, M = eng.nbf, 3 * b.natom
    Dt = torch.from_numpy(density(n, 1)).cuda()
    cols = np.stack([eng.grad_adjoint_jvp(Dt, np.eye(M)[i], 1.0, -0.5).cpu().numpy() for i in range(M)], axis=1)
    v = np.random.default_rng(5).normal(size=M)
    hv = eng.grad_adjoint_jvp(Dt, v, 1.0, -0.5).cpu().numpy()
    assert np.abs(cols @ v - hv).max() < 1e-10 * max(1.0, np.abs(hv).max())
    h, i = 1e-4, M - 2
    X = b.atom_coords().reshape(-1)
    gp = _engine(b.with_coords((X + h * np.eye(M)[i]).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5)
    gm = _engine(b.with_coords((X - h * np.eye(M)[i]).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5)
    fd = ((gp - gm) / (2 * h)).cpu().numpy()
    assert np.abs(cols[:, i] - fd).max() < 1e-6 * max(1.0, np.abs(fd).max())


@pytest.mark.parametrize("seed", [0, 2])
def test_hvp_with_d_and_f(oracle_lib, seed):
    """Hessian-vector product of sum Gamma G (Gamma fixed) with d and f shells:
    against the oracle's order-2 tensor contracted with Gamma and v, and against
    central differences of the adjoint gradient (h = 1e-4 bohr, 1e-6 relative)."""
    b = f_synthetic(seed, natom=2, heavy=(0, 2), kmax=2)
    eng = _engine(b, 1e-12)
    n, M = eng.nbf, 3 * b.natom
    D = density(n, seed)
    Dt = torch.from_numpy(D).cuda()
    v = np.random.default_rng(seed).normal(size=M)
    hv = eng.grad_adjoint_jvp(Dt, v, 1.0, -0.5).cpu().numpy()
    H = _unpack_pairs(oracle_lib.eri_deriv2(oracle_lib.OracleBasis(b), 1e-12).reshape(-1, n, n, n, n), M)
    Gam = np.einsum("ij,kl->ijkl", D, D) - 0.5 * np.einsum("ik,jl->ijkl", D, D)
    HG = np.einsum("abijkl,ijkl->ab", H, Gam)
    assert np.abs(hv - HG @ v).max() < 1e-9 * max(1.0, np.abs(HG).max())
    h = 1e-4
    X = b.atom_coords().reshape(-1)
    gp = _engine(b.with_coords((X + h * v).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5).cpu().numpy()
    gm = _engine(b.with_coords((X - h * v).reshape(-1, 3)), 1e-12).grad_adjoint(Dt, 1.0, -0.5).cpu().numpy()
    fd = (gp - gm) / (2 * h)
    assert np.abs(hv - fd).max() < 1e-6 * max(1.0, np.abs(fd).max())


def test_rys_engine_on_l2_classes(oracle_lib):
    """The Rys engine forced on every l <= 2 class (plain and gradient) reproduces
    the oracle, like the Obara-Saika engines it stands beside."""
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0)
    b = synthetic_molecule(spec, 1)[1]
    eng = _engine(b, 1e-12)
    for c in eng.class_info():
        eng.set_engine(c["cls"], plain="rys", deriv="rys")
    assert all(v[0] == "rys" and v[2] == "rys" for v in eng.engine_config().values())
    ob = oracle_lib.OracleBasis(b)
    G = eng.eri().cpu().numpy()
    assert np.abs(G - oracle_lib.compute_2e_int(ob, 1e-12)).max() < ATOL
    D = density(eng.nbf, 1)
    g = eng.grad_adjoint(torch.from_numpy(D).cuda(), 1.0, -0.5).cpu().numpy()
    gr = oracle_lib.grad_contract(ob, 1e-12, D, 1.0, -0.5)
    assert np.abs(g - gr).max() < ATOL_G * max(1.0, np.abs(gr).max())


@pytest.mark.parametrize("images", [False, True])
def test_plain_tiled_gradient_equals_adjoint(oracle_lib, images):
    """The plain path (derivative integrals materialised tile by tile as (3N, tile)
    tensors -- with images, the reference tensor's elements -- then contracted with
    Gamma) equals the adjoint gradient and the oracle, with warp and Rys engines
    and tiles smaller than a class."""
    b = f_synthetic(1)
    eng = _engine(b, 1e-12)
    D = torch.from_numpy(density(eng.nbf, 1)).cuda()
    ga = eng.grad_adjoint(D, 1.0, -0.5).cpu().numpy()
    gp = eng.grad_plain(D, 1.0, -0.5, images=images, tile_bytes=3 * b.natom * 8 * 5000).cpu().numpy()
    gr = oracle_lib.grad_contract(oracle_lib.OracleBasis(b), 1e-12, D.cpu().numpy(), 1.0, -0.5)
    scale = max(1.0, np.abs(gr).max())
    assert np.abs(gp - ga).max() < ATOL_G * scale
    assert np.abs(gp - gr).max() < ATOL_G * scale


@pytest.mark.parametrize("k", [3, 4])
def test_h2o_high_order_deriv_core(oracle_lib, k):
    """Orders 3 and 4 (the reference reaches them by nested jacfwd,
    quax/core.py:93-97): the dense tensor (C(3N+k-1, k), n, n, n, n) and one slice
    against the oracle's order-k tensor with the reference's cartesian-product
    semantics.  Tolerance HIGH_ORDER_TOL[k] x max(1, max |value|), set by the
    oracle's own error: against 40-digit values of the worst elements, the oracle
    is off by 3.1e-10 (order 3) and 3.3e-7 (order 4), the GPU by 1.0e-11 and 4.1e-9
    (an order-k derivative carries factors up to (2 alpha)^k, alpha = 130.7 for the
    oxygen 1s here)."""
    from quax_b200.basis import build_basis, h2o_config1
    from quax_b200.utils import get_deriv_vec_idx

    b = build_basis(h2o_config1(), "sto-3g")
    eng = _engine(b, 1e-14)
    ob = oracle_lib.OracleBasis(b)
    d = eng.eri_deriv_core(k).cpu().numpy()
    ref = oracle_lib.eri_derivk(ob, 1e-14, k)
    scale = max(1.0, np.abs(ref).max())
    assert d.shape == ref.shape
    err = np.abs(d - ref).max()
    assert err < HIGH_ORDER_TOL[k] * scale, err
    dv = np.zeros(9, dtype=int)
    dv[1] += 1
    dv[4] += k - 2
    dv[8] += 1
    s = eng.eri_deriv(dv).cpu().numpy()
    assert np.abs(s - ref[get_deriv_vec_idx(dv)]).max() < HIGH_ORDER_TOL[k] * scale


def test_order3_with_d_shells(oracle_lib):
    """Order 3 with d shells (every l <= 2 class has an order-3 program); the
    worst element's oracle error is 1.2e-8 against its 40-digit value (GPU 3.4e-9)."""
    spec = SyntheticSpec(natom=2, box=3.0, min_sep=1.2, kmax=2, exp_lo=0.2, exp_hi=20.0, heavy_ls=(0, 1, 2),
                         h_ls=(0, 1))
    b = synthetic_molecule(spec, 6)[1]
    eng = _engine(b, 1e-12)
    d = eng.eri_deriv_core(3).cpu().numpy()
    ref = oracle_lib.eri_derivk(oracle_lib.OracleBasis(b), 1e-12, 3)
    err = np.abs(d - ref).max()
    assert err < HIGH_ORDER_TOL[3] * max(1.0, np.abs(ref).max()), err
