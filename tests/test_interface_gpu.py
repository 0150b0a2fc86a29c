"""The reference-shaped API (libint_interface module, TEI) on the GPU, against the
oracle; the adjoint-backed autograd gradient against central finite differences
(step 1e-4 bohr, as the gradient configuration prescribes)."""
import os

import numpy as np
import pytest
import torch

from quax_b200.basis import Molecule, SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu


@pytest.fixture()
def h2o_xyz(tmp_path):
    p = str(tmp_path / "geom.xyz")
    h2o_config1().to_xyz(p)
    return p


def test_libint_interface_roundtrip(oracle_lib, h2o_xyz):
    from quax_b200.integrals import libint_interface as li

    li.initialize(h2o_xyz, "sto-3g", "sto-3g", "sto-3g", "sto-3g", 1e-14)
    b = build_basis(Molecule.from_xyz(h2o_xyz), "sto-3g")
    ob = oracle_lib.OracleBasis(b)
    G = li.compute_2e_int("eri", 0.0)
    assert G.shape == (7**4,)
    assert np.abs(G - oracle_lib.compute_2e_int(ob, 1e-14).reshape(-1)).max() < 1e-12
    dv = [0] * 9
    dv[5] = 1
    d = li.compute_2e_deriv("eri", 0.0, dv)
    assert np.abs(d - oracle_lib.eri_deriv1(ob, 1e-14, deriv_idx=5).reshape(-1)).max() < 1e-11
    core = li.eri_deriv_core(1)
    assert core.shape == (9 * 7**4,)
    assert np.abs(core - oracle_lib.eri_deriv1(ob, 1e-14).reshape(-1)).max() < 1e-11
    with pytest.raises(ValueError):
        li.compute_2e_int("coulomb", 0.0)
    with pytest.raises(NotImplementedError):
        li.compute_2e_int("f12", 1.0)
    with pytest.raises(ValueError):
        li.compute_2e_deriv("eri", 0.0, [1, 0])
    assert li.generate_multi_index_lookup(12, 1)[-1] == [11]
    li.finalize()


def test_tei_jvp_and_batch_semantics():
    from quax_b200.integrals.tei import TEI

    b = build_basis(h2o_config1(), "sto-3g")
    core = TEI(b, max_deriv_order=1, mode="core")
    f12 = TEI(b, max_deriv_order=1, mode="f12", engine=core.engine)
    geom = torch.zeros(9)
    rows = torch.eye(9, dtype=torch.int64)
    G, dG = core.eri_jvp((geom,), (rows[4],))
    assert torch.equal(G, core.eri(geom))
    assert (dG - f12.eri_deriv(geom, rows[4])).abs().max().item() < 1e-12
    batch, axis = core.eri_deriv_batch((geom, rows), (None, 0))  # tei.py:403-411's signature
    assert axis == 0 and batch.shape == (9, 7, 7, 7, 7)
    assert (batch - core.eri_derivatives[0]).abs().max().item() == 0.0


def test_tei_reference_constructor(tmp_path, oracle_lib):
    """TEI(basis1, basis2, basis3, basis4, xyz_path, max_deriv_order, options, mode)
    as quax/methods/ints.py builds it: libint_interface initialised from the xyz
    file first, then the TEI on the module's state; slices equal the oracle's."""
    from quax_b200.basis import Molecule
    from quax_b200.integrals import libint_interface as li
    from quax_b200.integrals.tei import TEI

    mol = h2o_config1()
    xyz = str(tmp_path / "h2o.xyz")
    mol.to_xyz(xyz)
    b = build_basis(Molecule.from_xyz(xyz, units="angstrom"), "sto-3g")
    ob = oracle_lib.OracleBasis(b)
    li.initialize(xyz, "sto-3g", "sto-3g", "sto-3g", "sto-3g", 1e-14)
    try:
        tei = TEI(b, b, b, b, xyz, 2, {"ints_tolerance": 1e-14}, "core")
        assert tei.engine is li.engine() and tei.nbf1 == 7
        dv = np.zeros(9, dtype=int)
        dv[4] = 1
        ref = oracle_lib.eri_deriv1(ob, 1e-14, deriv_idx=4)
        assert np.abs(tei.eri_deriv(torch.zeros(9), dv).cpu().numpy() - ref).max() < 1e-11
        dv[7] = 1
        from quax_b200.utils import get_deriv_vec_idx

        ref2 = oracle_lib.eri_deriv2(ob, 1e-14, pair_idx=get_deriv_vec_idx(dv))
        assert np.abs(tei.eri_deriv(torch.zeros(9), dv).cpu().numpy() - ref2).max() < 1e-11
        assert np.abs(tei.eri(torch.zeros(9)).cpu().numpy() - oracle_lib.compute_2e_int(ob, 1e-14)).max() < 1e-12
    finally:
        li.finalize()
    # without an initialised module the TEI initialises it from the xyz file and basis name
    tei = TEI("sto-3g", "sto-3g", "sto-3g", "sto-3g", xyz, 0, {}, "f12")
    try:
        dv = np.zeros(9, dtype=int)
        dv[2] = 1
        ref = oracle_lib.eri_deriv1(ob, 1e-14, deriv_idx=2)
        assert np.abs(tei.eri_deriv(None, dv).cpu().numpy() - ref).max() < 1e-11
    finally:
        li.finalize()


def test_adjoint_autograd_against_finite_differences():
    from quax_b200.integrals.engine import EriEngine
    from quax_b200.integrals.tei import two_electron_energy

    spec = SyntheticSpec(natom=3, box=4.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=30.0)
    mol, b = synthetic_molecule(spec, 3)
    n = b.nbf()
    rng = np.random.default_rng(5)
    C = rng.normal(0, 1 / np.sqrt(n), size=(n, n // 4))
    D = torch.from_numpy(C @ C.T).cuda()
    geom = torch.tensor(mol.coords.reshape(-1), dtype=torch.float64, requires_grad=True)
    eng = EriEngine(b, 1e-14)
    E = two_electron_energy(geom, D, eng)
    (g,) = torch.autograd.grad(E, geom)
    h = 1e-4
    fd = np.zeros(3 * b.natom)
    for nu in range(3 * b.natom):
        Es = []
        for s in (+1, -1):
            c = mol.coords.copy()
            c.flat[nu] += s * h
            e2 = EriEngine(b.with_coords(c), 1e-14)
            Es.append(float(two_electron_energy(geom.detach(), D, e2)))
            e2.close()
        fd[nu] = (Es[0] - Es[1]) / (2 * h)
    assert np.abs(g.cpu().numpy() - fd).max() < 1e-6 * max(1.0, np.abs(fd).max())


def test_disk_mode_roundtrip(tmp_path, monkeypatch):
    """compute_2e_deriv_disk / oei_deriv_disk write the reference's datasets
    (derivative index last; .npz where h5py is absent) and TEI(mode="disk") reads
    the slices back."""
    from quax_b200.integrals import libint_interface as li
    from quax_b200.integrals.tei import TEI

    monkeypatch.chdir(tmp_path)
    mol = h2o_config1()
    b = build_basis(mol, "sto-3g")
    li.initialize_basis(b, 1e-14, charges=mol.Z)
    try:
        path = li.compute_2e_deriv_disk("eri", 0.0, 2)
        n = b.nbf()
        d1 = li.read_dataset("eri_derivs", f"eri_{n}_{n}_{n}_{n}_deriv1")
        d2 = li.read_dataset("eri_derivs", f"eri_{n}_{n}_{n}_{n}_deriv2")
        assert d1.shape == (n, n, n, n, 9) and d2.shape == (n, n, n, n, 45)
        core = li.engine().eri_deriv_core(1).cpu().numpy()
        assert np.abs(np.moveaxis(d1, -1, 0) - core).max() == 0.0
        tei = TEI(b, mode="disk", engine=li.engine())
        dv = np.zeros(9, dtype=int)
        dv[3] = 1
        dv[7] = 1
        from quax_b200.utils import get_deriv_vec_idx

        assert np.abs(tei.eri_deriv(None, dv).cpu().numpy() - d2[..., get_deriv_vec_idx(dv)]).max() == 0.0
        li.oei_deriv_disk(1)
        s1 = li.read_dataset("oei_derivs", f"overlap_{n}_{n}_deriv1")
        assert s1.shape == (n, n, 9)
        assert path.startswith("eri_derivs.")
        # without eri_derivs the per-slice file eri_partials is read (tei.py:164-168):
        # datasets eri_n_n_n_n_deriv<k>_<flattened index>, four-dimensional
        os.remove(path)
        idx = get_deriv_vec_idx(dv)
        np.savez("eri_partials.npz", **{f"eri_{n}_{n}_{n}_{n}_deriv2_{idx}": d2[..., idx]})
        assert np.abs(tei.eri_deriv(None, dv).cpu().numpy() - d2[..., idx]).max() == 0.0
        os.remove("eri_partials.npz")
        with pytest.raises(FileNotFoundError):
            tei.eri_deriv(None, dv)
    finally:
        li.finalize()
