"""GPU one-electron integrals (qx_oei, qx_oei_deriv_core) against the host
McMurchie-Davidson implementation (quax_b200.oei, separate code) and against
central differences of the GPU integrals themselves.  Tolerances: integrals 1e-12
absolute, derivatives 1e-11 absolute, finite differences (h = 1e-4 bohr) 1e-6."""
import numpy as np
import pytest
import torch

from quax_b200.basis import SyntheticSpec, build_basis, h2o_config1, synthetic_molecule
from quax_b200.oei import one_electron

pytestmark = pytest.mark.gpu


def _cases():
    mol = h2o_config1()
    yield "h2o", mol.Z, build_basis(mol, "sto-3g")
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0)
    for seed in (0, 2):
        m, b = synthetic_molecule(spec, seed)
        yield f"syn{seed}", m.Z, b


@pytest.mark.parametrize("case", ["h2o", "syn0", "syn2"])
def test_oei_matches_host(case):
    from quax_b200.integrals.engine import EriEngine

    name, Z, b = next(c for c in _cases() if c[0] == case)
    eng = EriEngine(b, 1e-12)
    eng.set_charges(Z)
    S, T, V = (x.cpu().numpy() for x in eng.oei())
    dS, dT, dV = (x.cpu().numpy() for x in eng.oei_deriv(1))
    hS, hT, hV, hdS, hdT, hdV = one_electron(b, Z, b.atom_coords(), deriv=True)
    for g, h in ((S, hS), (T, hT), (V, hV)):
        assert np.abs(g - h).max() < 1e-12 * max(1.0, np.abs(h).max())
    for g, h in ((dS, hdS), (dT, hdT), (dV, hdV)):
        assert np.abs(g - h).max() < 1e-11 * max(1.0, np.abs(h).max())
    # translational invariance of every derivative tensor
    for d in (dS, dT, dV):
        assert np.abs(d.reshape(-1, 3, *d.shape[1:]).sum(axis=0)).max() < 1e-10


def test_oei_deriv_finite_differences():
    from quax_b200.integrals.engine import EriEngine

    _, Z, b = next(c for c in _cases() if c[0] == "syn2")
    eng = EriEngine(b, 1e-12)
    eng.set_charges(Z)
    d = [x.cpu().numpy() for x in eng.oei_deriv(1)]
    X = b.atom_coords().reshape(-1)
    h = 1e-4
    for nu in (0, 4, 3 * b.natom - 1):
        vals = []
        for sgn in (1, -1):
            Y = X.copy()
            Y[nu] += sgn * h
            e = EriEngine(b.with_coords(Y.reshape(-1, 3)), 1e-12)
            e.set_charges(Z)
            vals.append([x.cpu().numpy() for x in e.oei()])
            e.close()
        for k in range(3):
            fd = (vals[0][k] - vals[1][k]) / (2 * h)
            assert np.abs(fd - d[k][nu]).max() < 1e-6 * max(1.0, np.abs(fd).max())


def test_oei_module_interface():
    from quax_b200.integrals import libint_interface as li

    mol = h2o_config1()
    b = build_basis(mol, "sto-3g")
    li.initialize_basis(b, 1e-14, charges=mol.Z)
    try:
        n = b.nbf()
        hS, hT, hV = one_electron(b, mol.Z, mol.coords)
        assert np.abs(li.compute_1e_int("overlap").reshape(n, n) - hS).max() < 1e-12
        assert np.abs(li.compute_1e_int("potential").reshape(n, n) - hV).max() < 1e-12
        dv = np.zeros(9, dtype=int)
        dv[4] = 1
        _, _, _, _, hdT, _ = one_electron(b, mol.Z, mol.coords, deriv=True)
        assert np.abs(li.compute_1e_deriv("kinetic", dv).reshape(n, n) - hdT[4]).max() < 1e-11
        core = li.oei_deriv_core(1)
        assert len(core) == 3 and core[0].size == 9 * n * n
        with pytest.raises(ValueError):
            li.compute_1e_int("dipole")
        with pytest.raises(NotImplementedError):
            li.oei_deriv_core(2)
    finally:
        li.finalize()
