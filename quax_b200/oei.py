"""One-electron integrals and their nuclear derivatives, on the host.

The reference gets S, T, V and their derivative tensors from Libint
(quax/integrals/libint_interface.cc:101-155, 231-483, 2403-2581; quax/integrals/oei.py).
The library computes them on the GPU (qx_oei, qx_oei_deriv_core); this host
version is the independent check the tests compare the GPU kernel with, and the
nuclear-repulsion term of the RHF driver.  FP64, McMurchie-Davidson scheme (Hermite expansion coefficients
E^{ij}_t and Hermite Coulomb integrals R_tuv; McMurchie & Davidson, J. Comput.
Phys. 26, 218 (1978)).  Derivatives use d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}
on both centres; the derivative with respect to a nucleus in V follows from
translational invariance of each nuclear term.  Intended for small molecules
(pure Python loops over shells, components and primitives).
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .basis import Basis, cart_components


def boys_host(nmax: int, T: float) -> np.ndarray:
    """F_0..F_nmax(T): series at the top order then downward recursion; for large T,
    erf and upward recursion (Helgaker, Jorgensen & Olsen, sec. 9.8)."""
    F = np.empty(nmax + 1)
    if T < 1e-14:
        return 1.0 / (2 * np.arange(nmax + 1) + 1)
    eT = math.exp(-T)
    if T < 45.0:
        term = 1.0 / (2 * nmax + 1)
        s = term
        k = 1
        while True:
            term *= 2.0 * T / (2 * nmax + 2 * k + 1)
            s += term
            k += 1
            if term < s * 1e-17 or k > 5000:
                break
        F[nmax] = eT * s
        for m in range(nmax, 0, -1):
            F[m - 1] = (2.0 * T * F[m] + eT) / (2 * m - 1)
    else:
        F[0] = 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
        for m in range(nmax):
            F[m + 1] = ((2 * m + 1) * F[m] - eT) / (2.0 * T)
    return F


def _E(i, j, t, Q, a, b, memo):
    if t < 0 or t > i + j or i < 0 or j < 0:
        return 0.0
    key = (i, j, t)
    if key in memo:
        return memo[key]
    p = a + b
    q = a * b / p
    if i == j == t == 0:
        r = math.exp(-q * Q * Q)
    elif j == 0:
        r = (_E(i - 1, j, t - 1, Q, a, b, memo) / (2 * p) - q * Q / a * _E(i - 1, j, t, Q, a, b, memo)
             + (t + 1) * _E(i - 1, j, t + 1, Q, a, b, memo))
    else:
        r = (_E(i, j - 1, t - 1, Q, a, b, memo) / (2 * p) + q * Q / b * _E(i, j - 1, t, Q, a, b, memo)
             + (t + 1) * _E(i, j - 1, t + 1, Q, a, b, memo))
    memo[key] = r
    return r


class _PrimPair:
    """Cached Hermite data of one primitive pair."""

    def __init__(self, a, b, A, B):
        self.a, self.b, self.A, self.B = a, b, A, B
        self.p = a + b
        self.P = (a * A + b * B) / self.p
        self.memo = [dict(), dict(), dict()]

    def E(self, d, i, j, t):
        return _E(i, j, t, self.A[d] - self.B[d], self.a, self.b, self.memo[d])

    def overlap(self, la, lb):
        if min(la) < 0 or min(lb) < 0:
            return 0.0
        s = (math.pi / self.p) ** 1.5
        for d in range(3):
            s *= self.E(d, la[d], lb[d], 0)
        return s

    def kinetic(self, la, lb):
        if min(la) < 0 or min(lb) < 0:
            return 0.0
        b = self.b
        tot = 0.0
        for d in range(3):
            def sh(k):
                y = list(lb)
                y[d] += k
                return tuple(y)
            j = lb[d]
            t = -2 * b * b * self.overlap(la, sh(2)) + b * (2 * j + 1) * self.overlap(la, lb)
            if j >= 2:
                t -= 0.5 * j * (j - 1) * self.overlap(la, sh(-2))
            tot += t
        return tot

    def nuclear(self, la, lb, C, Z):
        """-Z <a| 1/|r-C| |b>."""
        if min(la) < 0 or min(lb) < 0:
            return 0.0
        p = self.p
        PC = self.P - C
        T = p * float(PC @ PC)
        L = sum(la) + sum(lb)
        F = boys_host(L, T)
        Rm = {}

        def R(t, u, v, n):
            if t < 0 or u < 0 or v < 0:
                return 0.0
            key = (t, u, v, n)
            if key in Rm:
                return Rm[key]
            if t == u == v == 0:
                r = (-2 * p) ** n * F[n]
            elif t == u == 0:
                r = (v - 1) * R(t, u, v - 2, n + 1) + PC[2] * R(t, u, v - 1, n + 1)
            elif t == 0:
                r = (u - 1) * R(t, u - 2, v, n + 1) + PC[1] * R(t, u - 1, v, n + 1)
            else:
                r = (t - 1) * R(t - 2, u, v, n + 1) + PC[0] * R(t - 1, u, v, n + 1)
            Rm[key] = r
            return r

        s = 0.0
        for t in range(la[0] + lb[0] + 1):
            ex = self.E(0, la[0], lb[0], t)
            for u in range(la[1] + lb[1] + 1):
                ey = self.E(1, la[1], lb[1], u)
                for v in range(la[2] + lb[2] + 1):
                    s += ex * ey * self.E(2, la[2], lb[2], v) * R(t, u, v, 0)
        return -Z * 2 * math.pi / p * s


def _shift(l3, d, k):
    y = list(l3)
    y[d] += k
    return tuple(y)


def one_electron(basis: Basis, Z, coords, deriv: bool = False):
    """S, T, V (n x n); with deriv=True also dS, dT, dV of shape (3N, n, n)."""
    if basis.pure:
        raise NotImplementedError("Cartesian shells only")
    n = basis.nbf()
    N3 = 3 * basis.natom
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    dS, dT, dV = (np.zeros((N3, n, n)) for _ in range(3)) if deriv else (None, None, None)
    coords = np.asarray(coords, float).reshape(-1, 3)
    s2bf = basis.shell2bf()
    for sa, A in enumerate(basis.shells):
        ca = A.norm_coefs()
        for sb, B in enumerate(basis.shells):
            if sb > sa:
                continue
            cb = B.norm_coefs()
            comps_a, comps_b = cart_components(A.l), cart_components(B.l)
            prims = [(ca[i] * cb[j], _PrimPair(A.exps[i], B.exps[j], np.asarray(A.center, float),
                                               np.asarray(B.center, float)))
                     for i in range(A.nprim) for j in range(B.nprim)]
            for ia, la in enumerate(comps_a):
                for ib, lb in enumerate(comps_b):
                    if sa == sb and ib > ia:
                        continue  # the (i, j) / (j, i) entries are set together below
                    s = t = v = 0.0
                    for w, pp in prims:
                        s += w * pp.overlap(la, lb)
                        t += w * pp.kinetic(la, lb)
                        for at in range(basis.natom):
                            v += w * pp.nuclear(la, lb, coords[at], Z[at])
                    i, j = s2bf[sa] + ia, s2bf[sb] + ib
                    S[i, j] = S[j, i] = s
                    T[i, j] = T[j, i] = t
                    V[i, j] = V[j, i] = v
                    if not deriv:
                        continue
                    for d in range(3):
                        gA = np.zeros(3)
                        gB = np.zeros(3)
                        vC = np.zeros(basis.natom)  # nuclear-position term, this direction
                        vA = vB = 0.0
                        for w, pp in prims:
                            a, b = pp.a, pp.b
                            up_a, dn_a = _shift(la, d, 1), _shift(la, d, -1)
                            up_b, dn_b = _shift(lb, d, 1), _shift(lb, d, -1)
                            gA[0] += w * (2 * a * pp.overlap(up_a, lb) - la[d] * pp.overlap(dn_a, lb))
                            gB[0] += w * (2 * b * pp.overlap(la, up_b) - lb[d] * pp.overlap(la, dn_b))
                            gA[1] += w * (2 * a * pp.kinetic(up_a, lb) - la[d] * pp.kinetic(dn_a, lb))
                            gB[1] += w * (2 * b * pp.kinetic(la, up_b) - lb[d] * pp.kinetic(la, dn_b))
                            for at in range(basis.natom):
                                C, Zc = coords[at], Z[at]
                                da = w * (2 * a * pp.nuclear(up_a, lb, C, Zc) - la[d] * pp.nuclear(dn_a, lb, C, Zc))
                                db = w * (2 * b * pp.nuclear(la, up_b, C, Zc) - lb[d] * pp.nuclear(la, dn_b, C, Zc))
                                vA += da
                                vB += db
                                vC[at] -= da + db
                        xa, xb = 3 * A.atom + d, 3 * B.atom + d
                        for arr, ga, gb in ((dS, gA[0], gB[0]), (dT, gA[1], gB[1]), (dV, vA, vB)):
                            arr[xa, i, j] += ga
                            arr[xb, i, j] += gb
                            if i != j:
                                arr[xa, j, i] += ga
                                arr[xb, j, i] += gb
                        for at in range(basis.natom):
                            dV[3 * at + d, i, j] += vC[at]
                            if i != j:
                                dV[3 * at + d, j, i] += vC[at]
    if deriv:
        return S, T, V, dS, dT, dV
    return S, T, V


def nuclear_repulsion(Z, coords, deriv: bool = False):
    coords = np.asarray(coords, float).reshape(-1, 3)
    E = 0.0
    g = np.zeros_like(coords)
    for i in range(len(Z)):
        for j in range(i):
            rij = coords[i] - coords[j]
            r = float(np.linalg.norm(rij))
            E += Z[i] * Z[j] / r
            g[i] -= Z[i] * Z[j] * rij / r**3
            g[j] += Z[i] * Z[j] * rij / r**3
    return (E, g.reshape(-1)) if deriv else E
