"""Spherical (pure) basis functions: GPU results through SphericalEngine against the
oracle's Cartesian tensor transformed on the host, J/K against the dense
spherical tensor, the adjoint gradient against central differences of
sum Gamma G_sph (h = 1e-4 bohr), and unit self-overlap of every spherical
function.  Tolerances as for the Cartesian tests."""
import numpy as np
import pytest
import torch

from quax_b200.basis import Basis, SyntheticSpec, synthetic_molecule

pytestmark = pytest.mark.gpu


def _pure(seed):
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0)
    m, b = synthetic_molecule(spec, seed)
    return m, Basis(b.shells, b.natom, True, b.name)


def test_spherical_eri_jk_oei(oracle_lib):
    from quax_b200.integrals.spherical import SphericalEngine, transform_matrix

    m, b = _pure(0)
    eng = SphericalEngine(b, 1e-12)
    n = eng.nbf
    assert n == b.nbf() < Basis(b.shells, b.natom, False).nbf()
    Tm = transform_matrix(b)
    Gc = oracle_lib.compute_2e_int(oracle_lib.OracleBasis(Basis(b.shells, b.natom, False)), 1e-12)
    Gs = np.einsum("ai,bj,ck,dl,ijkl->abcd", Tm, Tm, Tm, Tm, Gc, optimize=True)
    G = eng.eri().cpu().numpy()
    assert np.abs(G - Gs).max() < 1e-12
    rng = np.random.default_rng(1)
    C = rng.normal(size=(n, 3))
    D = C @ C.T / n
    J, K = (x.cpu().numpy() for x in eng.jk(torch.from_numpy(D)))
    assert np.abs(J - np.einsum("ijkl,kl->ij", Gs, D)).max() < 1e-11
    assert np.abs(K - np.einsum("ikjl,kl->ij", Gs, D)).max() < 1e-11
    eng.set_charges(m.Z)
    S, _, _ = eng.oei()
    assert np.abs(np.diag(S.cpu().numpy()) - 1.0).max() < 1e-12
    blocks = eng.eri_unique()
    assert all(t.shape[:4] == tuple(2 * l + 1 for l in k) for k, t in blocks.items())


def test_spherical_gradient_finite_differences():
    from quax_b200.integrals.spherical import SphericalEngine

    m, b = _pure(2)
    eng = SphericalEngine(b, 1e-12)
    n = eng.nbf
    rng = np.random.default_rng(3)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, 3))
    D = torch.from_numpy(C @ C.T).cuda()
    g = eng.grad_adjoint(D, 1.0, -0.5).cpu().numpy()

    def energy(X):
        e = SphericalEngine(b.with_coords(X.reshape(-1, 3)), 1e-12)
        G = e.eri()
        E = torch.einsum("ijkl,ij,kl->", G, D, D) - 0.5 * torch.einsum("ijkl,ik,jl->", G, D, D)
        e.close()
        return float(E)

    X = b.atom_coords().reshape(-1)
    h = 1e-4
    for nu in (0, 5, 3 * b.natom - 1):
        Xp, Xm = X.copy(), X.copy()
        Xp[nu] += h
        Xm[nu] -= h
        fd = (energy(Xp) - energy(Xm)) / (2 * h)
        assert abs(fd - g[nu]) < 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("f_shell", [False, True])
def test_spherical_unique_blocks_device_transform(f_shell):
    """The device transform of the unique blocks (qx_cart2sph_block, sparse
    coefficients, one thread per value) against four batched-GEMM quarter
    transforms of the same Cartesian blocks (1e-13: two FP64 summation orders),
    on two calls in a row (its buffers are reused), with d and f shells."""
    from quax_b200.integrals.spherical import SphericalEngine

    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0, f_shell=f_shell)
    _, bc = synthetic_molecule(spec, 4)
    eng = SphericalEngine(Basis(bc.shells, bc.natom, True, bc.name), 1e-12)
    ref = eng.eri_unique_gemm()
    assert not f_shell or any(3 in k for k in ref)
    for _ in range(2):
        got = eng.eri_unique()
        assert got.keys() == ref.keys()
        for k in ref:
            assert got[k].shape == ref[k].shape
            assert (got[k] - ref[k]).abs().max().item() < 1e-13, k
    eng.close()


def test_cart2sph_block_errors():
    import ctypes as C

    from quax_b200.integrals import _lib
    from quax_b200.integrals.spherical import _T_PACKED

    lib = _lib.load()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(x.data_ptr())
    for l4, nq, rc in (((4, 0, 0, 0), 1, -3), ((0, 0, 0, 0), -1, -1), ((1, 0, 0, 0), 0, 0)):
        assert lib.qx_cart2sph_block(p, p, _lib.iptr(np.array(l4, dtype=np.int32)), nq, _lib.dptr(_T_PACKED),
                                     None) == rc
