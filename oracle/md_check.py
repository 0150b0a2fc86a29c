"""Independent second algorithm: McMurchie-Davidson ERIs in pure Python.

TEST INFRASTRUCTURE ONLY.  Used to pin the C oracle (Obara-Saika/HGP) on small
cases with an algorithm that shares no code with it:
  McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978): Hermite expansion
  coefficients E^{ij}_t and Hermite Coulomb integrals R_{tuv}; the Boys function
  is taken from mpmath (incomplete gamma, 30 digits), not from either C library.
Cartesian ordering and normalisation follow quax_b200.basis (Libint convention).
Derivatives use d/dA_x g_a = 2 a g_{a+1x} - a_x g_{a-1x} on top of the MD
integral, which is independent of the oracle's recurrences.
"""
from __future__ import annotations

import math
from functools import lru_cache

import mpmath
import numpy as np

from quax_b200.basis import cart_components, normalize_contraction

mpmath.mp.dps = 30


@lru_cache(maxsize=None)
def _boys(n: int, T: float) -> float:
    if T < 1e-15:
        return 1.0 / (2 * n + 1)
    Tm = mpmath.mpf(T)
    return float(mpmath.gammainc(n + mpmath.mpf(0.5), 0, Tm) / (2 * Tm ** (n + mpmath.mpf(0.5))))


def _E(i, j, t, Qx, a, b, memo):
    key = (i, j, t)
    if key in memo:
        return memo[key]
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        r = 0.0
    elif i == j == t == 0:
        r = math.exp(-q * Qx * Qx)
    elif j == 0:
        r = (1 / (2 * p)) * _E(i - 1, j, t - 1, Qx, a, b, memo) - (q * Qx / a) * _E(i - 1, j, t, Qx, a, b, memo) + (
            t + 1
        ) * _E(i - 1, j, t + 1, Qx, a, b, memo)
    else:
        r = (1 / (2 * p)) * _E(i, j - 1, t - 1, Qx, a, b, memo) + (q * Qx / b) * _E(i, j - 1, t, Qx, a, b, memo) + (
            t + 1
        ) * _E(i, j - 1, t + 1, Qx, a, b, memo)
    memo[key] = r
    return r


def _R(t, u, v, n, p, PC, memo):
    key = (t, u, v, n)
    if key in memo:
        return memo[key]
    if t < 0 or u < 0 or v < 0:
        return 0.0
    if t == u == v == 0:
        T = p * float(PC @ PC)
        r = (-2 * p) ** n * _boys(n, T)
    elif t == u == 0:
        r = (v - 1) * _R(t, u, v - 2, n + 1, p, PC, memo) + PC[2] * _R(t, u, v - 1, n + 1, p, PC, memo)
    elif t == 0:
        r = (u - 1) * _R(t, u - 2, v, n + 1, p, PC, memo) + PC[1] * _R(t, u - 1, v, n + 1, p, PC, memo)
    else:
        r = (t - 1) * _R(t - 2, u, v, n + 1, p, PC, memo) + PC[0] * _R(t - 1, u, v, n + 1, p, PC, memo)
    memo[key] = r
    return r


def prim_eri(la3, lb3, lc3, ld3, a, b, c, d, A, B, Cc, D):
    """Primitive (unnormalised) Cartesian ERI via MD."""
    p, q = a + b, c + d
    P = (a * A + b * B) / p
    Q = (c * Cc + d * D) / q
    alpha = p * q / (p + q)
    PQ = P - Q
    Eab = [dict() for _ in range(3)]
    Ecd = [dict() for _ in range(3)]
    Rm = {}
    tot = 0.0
    for t in range(la3[0] + lb3[0] + 1):
        e1 = _E(la3[0], lb3[0], t, A[0] - B[0], a, b, Eab[0])
        for u in range(la3[1] + lb3[1] + 1):
            e2 = _E(la3[1], lb3[1], u, A[1] - B[1], a, b, Eab[1])
            for v in range(la3[2] + lb3[2] + 1):
                e3 = _E(la3[2], lb3[2], v, A[2] - B[2], a, b, Eab[2])
                for tau in range(lc3[0] + ld3[0] + 1):
                    f1 = _E(lc3[0], ld3[0], tau, Cc[0] - D[0], c, d, Ecd[0])
                    for nu in range(lc3[1] + ld3[1] + 1):
                        f2 = _E(lc3[1], ld3[1], nu, Cc[1] - D[1], c, d, Ecd[1])
                        for phi in range(lc3[2] + ld3[2] + 1):
                            f3 = _E(lc3[2], ld3[2], phi, Cc[2] - D[2], c, d, Ecd[2])
                            tot += (
                                e1 * e2 * e3 * f1 * f2 * f3 * (-1) ** (tau + nu + phi)
                                * _R(t + tau, u + nu, v + phi, 0, alpha, PQ, Rm)
                            )
    return 2 * math.pi**2.5 / (p * q * math.sqrt(p + q)) * tot


def _shift(l3, i, s):
    y = list(l3)
    y[i] += s
    return tuple(y)


def shell_quartet(shells, deriv=False):
    """Contracted Cartesian quartet block for 4 quax_b200.basis.Shell objects.

    deriv=False -> array (n1,n2,n3,n4); deriv=True -> (12,n1,n2,n3,n4) with the
    Libint first-derivative buffer order 3*centre + xyz.
    """
    comps = [cart_components(s.l) for s in shells]
    coefs = [s.norm_coefs() for s in shells]
    cen = [np.asarray(s.center, float) for s in shells]
    shape = tuple(len(c) for c in comps)
    out = np.zeros(((12,) if deriv else ()) + shape)
    for i1, c1 in enumerate(comps[0]):
        for i2, c2 in enumerate(comps[1]):
            for i3, c3 in enumerate(comps[2]):
                for i4, c4 in enumerate(comps[3]):
                    ls = [c1, c2, c3, c4]
                    acc = np.zeros(12) if deriv else 0.0
                    for p1, a in enumerate(shells[0].exps):
                        for p2, b in enumerate(shells[1].exps):
                            for p3, c in enumerate(shells[2].exps):
                                for p4, d in enumerate(shells[3].exps):
                                    w = coefs[0][p1] * coefs[1][p2] * coefs[2][p3] * coefs[3][p4]
                                    ex = [a, b, c, d]
                                    if not deriv:
                                        acc += w * prim_eri(*ls, a, b, c, d, *cen)
                                        continue
                                    for ctr in range(4):
                                        for x in range(3):
                                            lp = list(ls)
                                            lp[ctr] = _shift(ls[ctr], x, +1)
                                            val = 2 * ex[ctr] * prim_eri(*lp, a, b, c, d, *cen)
                                            if ls[ctr][x] > 0:
                                                lm = list(ls)
                                                lm[ctr] = _shift(ls[ctr], x, -1)
                                                val -= ls[ctr][x] * prim_eri(*lm, a, b, c, d, *cen)
                                            acc[3 * ctr + x] += w * val
                    if deriv:
                        out[:, i1, i2, i3, i4] = acc
                    else:
                        out[i1, i2, i3, i4] = acc
    return out


def overlap_xl(shell) -> float:
    """<x^l|x^l> of a contracted shell, Libint normalisation applied (should be 1)."""
    c = shell.norm_coefs()
    l = shell.l
    tot = 0.0
    for p, a in enumerate(shell.exps):
        for q, b in enumerate(shell.exps):
            g = a + b
            sx = math.sqrt(math.pi / g) * np.prod(np.arange(2 * l - 1, 0, -2, dtype=float)) / (2 * g) ** l
            tot += c[p] * c[q] * sx * (math.pi / g)
    return tot


def normalized(shell):
    return normalize_contraction(shell.l, shell.exps, shell.coefs)


def shell_quartet_deriv2(shells):
    """(12, 12, n1, n2, n3, n4) second derivatives by McMurchie-Davidson, applying the
    derivative identity on all four centres directly (no translational invariance)."""
    comps = [cart_components(s.l) for s in shells]
    coefs = [s.norm_coefs() for s in shells]
    cen = [np.asarray(s.center, float) for s in shells]
    shape = tuple(len(c) for c in comps)
    out = np.zeros((12, 12) + shape)
    for i1, c1 in enumerate(comps[0]):
        for i2, c2 in enumerate(comps[1]):
            for i3, c3 in enumerate(comps[2]):
                for i4, c4 in enumerate(comps[3]):
                    ls = [c1, c2, c3, c4]
                    acc = np.zeros((12, 12))
                    for p1, a in enumerate(shells[0].exps):
                        for p2, b in enumerate(shells[1].exps):
                            for p3, c in enumerate(shells[2].exps):
                                for p4, d in enumerate(shells[3].exps):
                                    w = coefs[0][p1] * coefs[1][p2] * coefs[2][p3] * coefs[3][p4]
                                    ex = [a, b, c, d]
                                    for P in range(12):
                                        X, i = divmod(P, 3)
                                        for Q in range(P, 12):
                                            Y, j = divmod(Q, 3)
                                            tot = 0.0
                                            for fx in (0, 1):
                                                for fy in (0, 1):
                                                    lp = [list(t) for t in ls]
                                                    coef = 1.0
                                                    if fx == 0:
                                                        coef *= 2 * ex[X]
                                                        lp[X][i] += 1
                                                    else:
                                                        coef *= -lp[X][i]
                                                        lp[X][i] -= 1
                                                    if coef == 0:
                                                        continue
                                                    if fy == 0:
                                                        coef *= 2 * ex[Y]
                                                        lp[Y][j] += 1
                                                    else:
                                                        coef *= -lp[Y][j]
                                                        lp[Y][j] -= 1
                                                    if coef == 0 or min(min(t) for t in lp) < 0:
                                                        continue
                                                    tot += coef * prim_eri(*[tuple(t) for t in lp], a, b, c, d, *cen)
                                            acc[P, Q] += w * tot
                    acc = np.triu(acc) + np.triu(acc, 1).T
                    out[:, :, i1, i2, i3, i4] = acc
    return out
