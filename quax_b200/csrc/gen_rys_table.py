#!/usr/bin/env python3
"""Generator of the Rys quadrature root/weight table (qx_rys_table.inc).

The Rys quadrature of a primitive electron-repulsion integral needs, for a Boys
argument T and n = floor(L/2) + 1 points, the nodes u_1..u_n in (0, 1) and the
weights w_1..w_n of the Gauss rule for the measure

    dmu_T(u) = exp(-T u) u^{-1/2} / 2 du   on [0, 1],

whose moments are the Boys function values: sum_r w_r u_r^m = F_m(T)
(M. Dupuis, J. Rys & H. F. King, J. Chem. Phys. 65, 111 (1976); J. Rys,
M. Dupuis & H. F. King, J. Comput. Chem. 4, 154 (1983)).

Method (published mathematics, written here):
  * F_m(T) = gamma(m + 1/2, T) / (2 T^{m + 1/2}) in 40-digit arithmetic (mpmath);
  * recurrence coefficients of the orthogonal polynomials from these moments by
    the Chebyshev algorithm (W. Gautschi, Orthogonal Polynomials: Computation and
    Approximation, Oxford 2004, sec. 2.1.7) -- ill-conditioned, which is why it
    runs in 40 digits;
  * nodes and weights as the eigen-decomposition of the n x n Jacobi matrix
    (G. H. Golub & J. H. Welsch, Math. Comp. 23, 221 (1969));
  * for T in [0, TMAX(n)) each node and weight is tabulated as a degree-13
    Chebyshev series on intervals [2i, 2i+2) (fit at the 14 Chebyshev points of
    each interval; measured relative error <= 3e-16 for the nodes, the weights
    and the moments sum w u^m, m < 2n);
  * for T >= TMAX(n): u_r = y_r / T, w_r = W_r / (2 sqrt(T)) with (y_r, W_r) the
    generalized Gauss-Laguerre rule of weight y^{-1/2} e^{-y} on [0, inf); TMAX(n)
    is the first even T where this rule reproduces F_0..F_{2n-1} to 2e-17
    relative (42 for n = 1 ... 80 for n = 9).

Output layout (double, hex-float literals):
  QX_RYS_TAB[off[n] + (interval * 2n + f) * 14 + k], f = 0..n-1 nodes, n..2n-1
  weights, k = Chebyshev degree; QX_RYS_ASYM_Y / _W[(n-1)*(n)/2 + r].

Run:  python gen_rys_table.py        (needs mpmath; about a minute on 8 cores)
"""
from __future__ import annotations

import os
from multiprocessing import get_context

import mpmath as mp

NMAX = 9
H = 2
DEG = 13
DPS = 40


def tmax_of(n: int) -> int:
    return {1: 42, 2: 48, 3: 54, 4: 58, 5: 62, 6: 68, 7: 72, 8: 76, 9: 80}[n]


def boys_moments(T, nmom):
    T = mp.mpf(T)
    if T == 0:
        return [mp.mpf(1) / (2 * m + 1) for m in range(nmom)]
    return [mp.gammainc(m + mp.mpf(0.5), 0, T) / (2 * T ** (m + mp.mpf(0.5))) for m in range(nmom)]


def recurrence(mu, N):
    """Chebyshev algorithm: alpha_k, beta_k (k < N) of the monic orthogonal
    polynomials of the measure with moments mu[0..2N-1]."""
    sig_prev = [mp.mpf(0)] * (2 * N)
    sig = [mu[l] for l in range(2 * N)]
    a = [mp.mpf(0)] * N
    b = [mp.mpf(0)] * N
    a[0] = mu[1] / mu[0]
    b[0] = mu[0]
    for k in range(1, N):
        sig_new = [mp.mpf(0)] * (2 * N)
        for l in range(k, 2 * N - k):
            sig_new[l] = sig[l + 1] - a[k - 1] * sig[l] - b[k - 1] * sig_prev[l]
        a[k] = sig_new[k + 1] / sig_new[k] - sig[k] / sig[k - 1]
        b[k] = sig_new[k] / sig[k - 1]
        sig_prev, sig = sig, sig_new
    return a, b


def gauss(a, b, n):
    """Golub-Welsch: nodes (ascending) and weights of the n-point rule."""
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = a[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(b[i + 1])
    E, Q = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in idx], [b[0] * Q[0, i] ** 2 for i in idx]


def _point(T):
    """Nodes and weights of every n at one T (shared moments)."""
    mp.mp.dps = DPS
    mu = boys_moments(T, 2 * NMAX)
    a, b = recurrence(mu, NMAX)
    return [gauss(a, b, n) for n in range(1, NMAX + 1)]


def main():
    mp.mp.dps = DPS
    nint_max = tmax_of(NMAX) // H
    N = DEG + 1
    xs = [mp.cos(mp.pi * (j + mp.mpf(0.5)) / N) for j in range(N)]
    pts = [i * H + (x + 1) * H / 2 for i in range(nint_max) for x in xs]
    with get_context("spawn").Pool(os.cpu_count() or 4) as pool:
        res = pool.map(_point, pts, chunksize=4)
    tab, off, nint = [], [], []
    for n in range(1, NMAX + 1):
        off.append(len(tab))
        ni = tmax_of(n) // H
        nint.append(ni)
        for i in range(ni):
            vals = [res[i * N + j][n - 1] for j in range(N)]  # (nodes, weights) at each Chebyshev point
            for f in range(2 * n):
                fv = [vals[j][0][f] if f < n else vals[j][1][f - n] for j in range(N)]
                for k in range(N):
                    s = sum(fv[j] * mp.cos(mp.pi * k * (j + mp.mpf(0.5)) / N) for j in range(N)) * 2 / N
                    if k == 0:
                        s /= 2
                    tab.append(float(s))
    ay, aw = [], []
    for n in range(1, NMAX + 1):
        mu = [mp.gamma(m + mp.mpf(0.5)) for m in range(2 * n)]
        a, b = recurrence(mu, n)
        y, W = gauss(a, b, n)
        ay += [float(v) for v in y]
        aw += [float(v) for v in W]
    here = os.path.dirname(os.path.abspath(__file__))
    L = ["// Generated by quax_b200/csrc/gen_rys_table.py -- do not edit by hand.",
         "// Rys quadrature nodes/weights: degree-13 Chebyshev series on T intervals [2i, 2i+2)",
         "// below QX_RYS_TMAX[n], generalized Gauss-Laguerre (alpha = -1/2) asymptotics above.",
         "#pragma once",
         f"#define QX_RYS_NMAX {NMAX}",
         f"#define QX_RYS_NCOEF {N}",
         "// T bound of the tabulated range and table offset (doubles), n = 0..QX_RYS_NMAX",
         "#define QX_RYS_TMAX_LIST 0, " + ", ".join(str(tmax_of(n)) for n in range(1, NMAX + 1)),
         "#define QX_RYS_OFF_LIST 0, " + ", ".join(str(o) for o in off),
         f"#define QX_RYS_TAB_SIZE {len(tab)}",
         "#define QX_RYS_TAB_DATA \\"]
    for i in range(0, len(tab), 4):
        L.append("    " + ", ".join(float.hex(v) for v in tab[i:i + 4]) + ", \\")
    L.append("")
    L.append(f"#define QX_RYS_ASYM_SIZE {len(ay)}")
    L.append("#define QX_RYS_ASYM_Y_DATA " + ", ".join(float.hex(v) for v in ay))
    L.append("#define QX_RYS_ASYM_W_DATA " + ", ".join(float.hex(v) for v in aw))
    with open(os.path.join(here, "qx_rys_table.inc"), "w") as fh:
        fh.write("\n".join(L) + "\n")
    print(f"wrote {len(tab)} coefficients, {len(ay)} asymptotic nodes")


if __name__ == "__main__":
    main()
