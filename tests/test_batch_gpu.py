"""Batched RHF (quax_b200.methods.batch): a batch of molecules of different sizes,
J/K of the whole batch in one CUDA graph.  Each molecule must reach the energy and
gradient of the single-molecule driver (1e-8 Eh, 1e-7 Eh/bohr: both SCFs converge
far below that in 40 iterations), and graph replay must reproduce the eager
results exactly up to summation order (1e-12)."""
import numpy as np
import pytest

from quax_b200.basis import Molecule, SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu


def _batch():
    mols, bases = [], []
    h2o = h2o_config1()
    mols.append(h2o)
    bases.append(build_basis(h2o, "sto-3g"))
    stretched = Molecule(h2o.Z.copy(), h2o.coords * 1.1, 0)
    mols.append(stretched)
    bases.append(build_basis(stretched, "sto-3g"))
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.3, kmax=3, exp_lo=0.2, exp_hi=30.0, charges=(1, 6))
    m, b = synthetic_molecule(spec, 4)
    mols.append(m)
    bases.append(b)
    return mols, bases


def test_batched_rhf_matches_single_molecule_driver():
    from quax_b200.methods.batch import BatchedRHF
    from quax_b200.methods.hartree_fock import rhf_gradient

    mols, bases = _batch()
    br = BatchedRHF(mols, bases, ints_tol=1e-12)
    E, t_jk = br.scf(iterations=40, use_graph=True)
    G = br.gradients()
    for k, (mol, b) in enumerate(zip(mols, bases)):
        E1, g1 = rhf_gradient(mol, b, ints_tol=1e-12, conv=1e-11)
        assert abs(E[k] - E1) < 1e-8
        assert np.abs(G[k] - g1).max() < 1e-7
    br.close()


def test_graph_replay_equals_eager():
    from quax_b200.methods.batch import BatchedRHF

    mols, bases = _batch()
    a = BatchedRHF(mols, bases, ints_tol=1e-12)
    Ea, _ = a.scf(iterations=6, use_graph=True)
    b = BatchedRHF(mols, bases, ints_tol=1e-12)
    Eb, _ = b.scf(iterations=6, use_graph=False)
    assert np.abs(np.array(Ea) - np.array(Eb)).max() < 1e-12
    a.close()
    b.close()


def test_incremental_screened_scf_matches_full_builds():
    from quax_b200.methods.batch import BatchedRHF

    mols, bases = _batch()
    full = BatchedRHF(mols, bases, ints_tol=1e-12)
    Ef, _ = full.scf(iterations=30, use_graph=True)
    inc = BatchedRHF(mols, bases, ints_tol=1e-12, incremental=1e-12, rebuild_every=8)
    Ei, _ = inc.scf(iterations=30, use_graph=True)
    assert np.abs(np.array(Ef) - np.array(Ei)).max() < 1e-8
    full.close()
    inc.close()
