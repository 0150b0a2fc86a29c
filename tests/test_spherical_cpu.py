"""Solid-harmonic coefficients (host only): every spherical function of a shell has
unit norm and the functions of a shell are orthogonal, with the Libint
normalisation of the Cartesian components (x^l of unit norm)."""
import numpy as np

from quax_b200.basis import Basis, Shell
from quax_b200.integrals.spherical import cart2sph, transform_matrix
from quax_b200.oei import one_electron


def test_solid_harmonics_orthonormal():
    shells = [Shell(2, np.array([1.3, 0.4]), np.array([0.6, 0.5]), np.zeros(3), 0),
              Shell(1, np.array([0.9]), np.array([1.0]), np.zeros(3), 0),
              Shell(0, np.array([2.0]), np.array([1.0]), np.zeros(3), 0)]
    S, _, _ = one_electron(Basis(shells, 1, False, "t"), np.array([1]), np.zeros((1, 3)))
    T = transform_matrix(Basis(shells, 1, True, "t"))
    # the blocks of one shell are orthonormal; different shells on one centre with
    # different l are orthogonal by symmetry
    Ss = T @ S @ T.T
    assert np.abs(np.diag(Ss) - 1.0).max() < 1e-12
    assert np.abs(Ss[:5, :5] - np.eye(5)).max() < 1e-12
    assert cart2sph(2).shape == (5, 6) and cart2sph(1).shape == (3, 3)
