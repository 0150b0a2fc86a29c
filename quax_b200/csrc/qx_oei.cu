// qx_oei.cu -- one-electron integrals S, T, V and their first nuclear derivatives.
//
// Replaces the one-electron part of the reference's Libint module
// (quax/integrals/libint_interface.cc:232-483 compute_1e_int, :650-788
// compute_1e_deriv, :2403-2579 oei_deriv_core) for the HF energy and gradient.
// O(n^2 natom) work next to the O(n^4) two-electron path, so the kernel favours
// simplicity: one warp per shell pair, one lane per Cartesian component pair,
// runtime angular momenta, primitive loops in registers.
//
// Method (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978); Obara & Saika,
// J. Chem. Phys. 84, 3963 (1986)):
//   overlap   1-D Obara-Saika recursion S(i+1,j) = PA S(i,j) + (i S(i-1,j) + j S(i,j-1))/2p
//             (and the j analogue with PB), S(0,0) = sqrt(pi/p);
//   kinetic   T_x(i,j) = -2 b^2 S(i,j+2) + b (2j+1) S(i,j) - j(j-1)/2 S(i,j-2);
//   nuclear   V = -Z_C (2 pi/p) sum_tuv E^x_t E^y_u E^z_v R_tuv(p, P-C) with the
//             Hermite coefficients E and the Hermite Coulomb integrals R;
//   derivatives d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x} (and for B); the
//             derivative of the nuclear term with respect to the nucleus C follows
//             from translational invariance of each term: d/dC = -(d/dA + d/dB).
// Every block is written for both (i,j) and (j,i) by the lane that owns it.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "quax_b200.h"
#include "qx_kernels.cuh"

namespace qx {

constexpr int OEI_LMAX = 3;               // shell AM the local tables are sized for
constexpr int OEI_NI = OEI_LMAX + 2;      // i up to la + 1
constexpr int OEI_NJ = OEI_LMAX + 4;      // j up to lb + 3 (kinetic of a B-derivative)
constexpr int OEI_NT = 2 * OEI_LMAX + 3;  // Hermite index t up to la + lb + 2
constexpr int OEI_LR = 2 * OEI_LMAX + 1;  // R_tuv with t + u + v <= la + lb + 1
constexpr int OEI_NR = (OEI_LR + 1) * (OEI_LR + 2) * (OEI_LR + 3) / 6;

struct OeiArgs {
    const PairInfo* pairs;
    int npair;
    const PrimPair* prims;
    const double* boys;
    const double* xyz;  // natom x 3 (bohr)
    const double* Z;    // natom
    int natom;
    long long n;
    double *S, *T, *V;     // n x n (may be null)
    double *dS, *dT, *dV;  // 3N x n x n (may be null)
};

__device__ __forceinline__ void cart_of(int l, int k, int& x, int& y, int& z) {
    // Libint standard order: lx from l down, then ly from l - lx down
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
            if (k == 0) {
                x = lx;
                y = ly;
                z = l - lx - ly;
                return;
            }
            --k;
        }
    x = y = z = 0;
}

__device__ __forceinline__ int ridx(int t, int u, int v) {
    // packed index of (t,u,v), t+u+v = s: offset of shell s plus position inside it
    const int s = t + u + v;
    const int k = u + v;
    return s * (s + 1) * (s + 2) / 6 + k * (k + 1) / 2 + v;
}

// 1-D overlaps S(i,j) for i <= ni, j <= nj (without the sqrt(pi/p) factor).
__device__ __forceinline__ void overlap_1d(double PA, double PB, double oo2p, int ni, int nj,
                                           double (&s)[OEI_NI][OEI_NJ]) {
    s[0][0] = 1.0;
    for (int i = 0; i < ni; ++i) s[i + 1][0] = PA * s[i][0] + (i ? i * oo2p * s[i - 1][0] : 0.0);
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i <= ni; ++i)
            s[i][j + 1] = PB * s[i][j] + oo2p * ((i ? i * s[i - 1][j] : 0.0) + (j ? j * s[i][j - 1] : 0.0));
}

// Kinetic 1-D factor acting on the ket index j.
__device__ __forceinline__ double kin_1d(const double (&s)[OEI_NI][OEI_NJ], int i, int j, double b) {
    double t = -2.0 * b * b * s[i][j + 2] + b * (2 * j + 1) * s[i][j];
    if (j >= 2) t -= 0.5 * j * (j - 1) * s[i][j - 2];
    return t;
}

// Hermite coefficients E^{ij}_t for i <= ni, j <= nj (1-D, without exp(-mu X^2)).
__device__ __forceinline__ void hermite_1d(double PA, double PB, double oo2p, int ni, int nj,
                                           double (&E)[OEI_NI][OEI_NI][OEI_NT]) {
    for (int i = 0; i <= ni; ++i)
        for (int j = 0; j <= nj; ++j)
            for (int t = 0; t < OEI_NT; ++t) E[i][j][t] = 0.0;
    E[0][0][0] = 1.0;
    for (int i = 0; i <= ni; ++i)
        for (int j = 0; j <= nj; ++j) {
            if (i == 0 && j == 0) continue;
            const bool up_i = i > 0;
            const int pi = up_i ? i - 1 : i, pj = up_i ? j : j - 1;
            const double X = up_i ? PA : PB;
            for (int t = 0; t <= i + j; ++t) {
                double v = X * E[pi][pj][t];
                if (t > 0) v += oo2p * E[pi][pj][t - 1];
                if (t + 1 <= pi + pj) v += (t + 1) * E[pi][pj][t + 1];
                E[i][j][t] = v;
            }
        }
}

__global__ void __launch_bounds__(128) k_oei(OeiArgs a) {
    const int lane = threadIdx.x & 31;
    const int pidx = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (pidx >= a.npair) return;
    const PairInfo P = a.pairs[pidx];
    const int la = P.l1, lb = P.l2;
    const int na = (la + 1) * (la + 2) / 2, nb = (lb + 1) * (lb + 2) / 2;
    const bool same = P.s1 == P.s2;
    const bool deriv = a.dS != nullptr;
    const double kfac = 5.914967172795613;  // sqrt(2) pi^(5/4), the factor in PrimPair::K
    for (int c = lane; c < na * nb; c += 32) {
        const int ia = c / nb, ib = c % nb;
        if (same && ib > ia) continue;  // the (ia, ib) lane writes (ib, ia) too
        int ax, ay, az, bx, by, bz;
        cart_of(la, ia, ax, ay, az);
        cart_of(lb, ib, bx, by, bz);
        double s = 0.0, t = 0.0, v = 0.0;
        double dsa[3] = {0, 0, 0}, dsb[3] = {0, 0, 0}, dta[3] = {0, 0, 0}, dtb[3] = {0, 0, 0};
        double dva[3] = {0, 0, 0}, dvb[3] = {0, 0, 0};
        const long long i0 = P.bf1 + ia, j0 = P.bf2 + ib;
        for (int k = 0; k < P.nprim; ++k) {
            const PrimPair pp = a.prims[P.prim_off + k];
            const double p = pp.zeta, al = pp.alpha, be = p - al, oo2p = pp.oo2z;
            const double w = pp.K * p / kfac;  // c_a c_b exp(-mu |AB|^2)
            const double PA[3] = {pp.PAx, pp.PAy, pp.PAz};
            const double PB[3] = {pp.PAx + P.ABx, pp.PAy + P.ABy, pp.PAz + P.ABz};
            const int la3[3] = {ax, ay, az}, lb3[3] = {bx, by, bz};
            // overlap and kinetic factors per dimension
            double S0[3], Sa[3], Sb[3], T0[3], Ta[3], Tb[3];
            const double rp = sqrt(3.14159265358979323846 / p);
            for (int d = 0; d < 3; ++d) {
                double tab[OEI_NI][OEI_NJ];
                const int ni = la3[d] + 1, nj = lb3[d] + 3;
                overlap_1d(PA[d], PB[d], oo2p, ni, nj, tab);
                const int i = la3[d], j = lb3[d];
                S0[d] = rp * tab[i][j];
                T0[d] = rp * kin_1d(tab, i, j, be);
                Sa[d] = rp * (2.0 * al * tab[i + 1][j] - (i ? i * tab[i - 1][j] : 0.0));
                Ta[d] = rp * (2.0 * al * kin_1d(tab, i + 1, j, be) - (i ? i * kin_1d(tab, i - 1, j, be) : 0.0));
                Sb[d] = rp * (2.0 * be * tab[i][j + 1] - (j ? j * tab[i][j - 1] : 0.0));
                Tb[d] = rp * (2.0 * be * kin_1d(tab, i, j + 1, be) - (j ? j * kin_1d(tab, i, j - 1, be) : 0.0));
            }
            s += w * S0[0] * S0[1] * S0[2];
            t += w * (T0[0] * S0[1] * S0[2] + S0[0] * T0[1] * S0[2] + S0[0] * S0[1] * T0[2]);
            if (deriv) {
                for (int d = 0; d < 3; ++d) {
                    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                    dsa[d] += w * Sa[d] * S0[d1] * S0[d2];
                    dsb[d] += w * Sb[d] * S0[d1] * S0[d2];
                    dta[d] += w * (Ta[d] * S0[d1] * S0[d2] + Sa[d] * (T0[d1] * S0[d2] + S0[d1] * T0[d2]));
                    dtb[d] += w * (Tb[d] * S0[d1] * S0[d2] + Sb[d] * (T0[d1] * S0[d2] + S0[d1] * T0[d2]));
                }
            }
            // nuclear attraction: Hermite expansion of the pair, one R table per nucleus
            double E[3][OEI_NI][OEI_NI][OEI_NT];
            for (int d = 0; d < 3; ++d) hermite_1d(PA[d], PB[d], oo2p, la3[d] + 1, lb3[d] + 1, E[d]);
            const int L = la + lb + (deriv ? 1 : 0);
            const double Px = pp.Px, Py = pp.Py, Pz = pp.Pz;
            for (int C = 0; C < a.natom; ++C) {
                const double XPC = Px - a.xyz[3 * C], YPC = Py - a.xyz[3 * C + 1], ZPC = Pz - a.xyz[3 * C + 2];
                const double T = p * (XPC * XPC + YPC * YPC + ZPC * ZPC);
                double F[2 * OEI_LMAX + 2];
                boys<2 * OEI_LMAX + 1>(T, a.boys, F);
                // R^{n}_{tuv}, n from L down to 0 (two packed buffers)
                double Rn[OEI_NR], Rm[OEI_NR];
                double m2p = 1.0;
                for (int q = 0; q < L; ++q) m2p *= -2.0 * p;
                for (int n = L; n >= 0; --n) {
                    const int top = L - n;
                    for (int s3 = 0; s3 <= top; ++s3)
                        for (int tt = s3; tt >= 0; --tt)
                            for (int uu = s3 - tt; uu >= 0; --uu) {
                                const int vv = s3 - tt - uu;
                                double r;
                                if (tt > 0)
                                    r = XPC * Rm[ridx(tt - 1, uu, vv)] + (tt > 1 ? (tt - 1) * Rm[ridx(tt - 2, uu, vv)] : 0.0);
                                else if (uu > 0)
                                    r = YPC * Rm[ridx(tt, uu - 1, vv)] + (uu > 1 ? (uu - 1) * Rm[ridx(tt, uu - 2, vv)] : 0.0);
                                else if (vv > 0)
                                    r = ZPC * Rm[ridx(tt, uu, vv - 1)] + (vv > 1 ? (vv - 1) * Rm[ridx(tt, uu, vv - 2)] : 0.0);
                                else
                                    r = m2p * F[n];
                                Rn[ridx(tt, uu, vv)] = r;
                            }
                    for (int q = 0; q < (top + 1) * (top + 2) * (top + 3) / 6; ++q) Rm[q] = Rn[q];
                    m2p /= -2.0 * p;
                }
                const double* R = Rm;  // R^{0}
                const double pre = -a.Z[C] * 2.0 * 3.14159265358979323846 / p * w;
                // Hermite sum for shifted component indices (sa, sb per dimension)
                auto hsum = [&](int ix, int jx, int iy, int jy, int iz, int jz) {
                    double acc = 0.0;
                    for (int tt = 0; tt <= ix + jx; ++tt) {
                        const double ex = E[0][ix][jx][tt];
                        if (ex == 0.0) continue;
                        for (int uu = 0; uu <= iy + jy; ++uu) {
                            const double exy = ex * E[1][iy][jy][uu];
                            if (exy == 0.0) continue;
                            for (int vv = 0; vv <= iz + jz; ++vv) acc += exy * E[2][iz][jz][vv] * R[ridx(tt, uu, vv)];
                        }
                    }
                    return acc;
                };
                v += pre * hsum(ax, bx, ay, by, az, bz);
                if (deriv) {
                    double ga[3], gb[3];
                    for (int d = 0; d < 3; ++d) {
                        int ia3[3] = {ax, ay, az}, ib3[3] = {bx, by, bz};
                        ia3[d] += 1;
                        double up = hsum(ia3[0], ib3[0], ia3[1], ib3[1], ia3[2], ib3[2]);
                        double dn = 0.0;
                        if (la3[d] > 0) {
                            ia3[d] -= 2;
                            dn = hsum(ia3[0], ib3[0], ia3[1], ib3[1], ia3[2], ib3[2]);
                            ia3[d] += 1;
                        } else {
                            ia3[d] -= 1;
                        }
                        ga[d] = pre * (2.0 * al * up - la3[d] * dn);
                        ib3[d] += 1;
                        up = hsum(ia3[0], ib3[0], ia3[1], ib3[1], ia3[2], ib3[2]);
                        dn = 0.0;
                        if (lb3[d] > 0) {
                            ib3[d] -= 2;
                            dn = hsum(ia3[0], ib3[0], ia3[1], ib3[1], ia3[2], ib3[2]);
                        }
                        gb[d] = pre * (2.0 * be * up - lb3[d] * dn);
                        dva[d] += ga[d];
                        dvb[d] += gb[d];
                    }
                    // nucleus C by invariance of this term
                    const long long nn = a.n * a.n;
                    for (int d = 0; d < 3; ++d) {
                        double* o = a.dV + (3LL * C + d) * nn;
                        o[i0 * a.n + j0] -= ga[d] + gb[d];
                        if (i0 != j0) o[j0 * a.n + i0] -= ga[d] + gb[d];
                    }
                }
            }
        }
        const long long n = a.n;
        auto put = [&](double* M, double x) {
            if (!M) return;
            M[i0 * n + j0] = x;
            M[j0 * n + i0] = x;
        };
        put(a.S, s);
        put(a.T, t);
        put(a.V, v);
        if (deriv) {
            const long long nn = n * n;
            auto add = [&](double* base, int atom, int d, double x) {
                double* o = base + (3LL * atom + d) * nn;
                o[i0 * n + j0] += x;
                if (i0 != j0) o[j0 * n + i0] += x;
            };
            for (int d = 0; d < 3; ++d) {
                add(a.dS, P.atom1, d, dsa[d]);
                add(a.dS, P.atom2, d, dsb[d]);
                add(a.dT, P.atom1, d, dta[d]);
                add(a.dT, P.atom2, d, dtb[d]);
                add(a.dV, P.atom1, d, dva[d]);
                add(a.dV, P.atom2, d, dvb[d]);
            }
        }
    }
}

}  // namespace qx

// Launch over every shell pair of a handle (one warp per pair); outputs zeroed by
// the caller where derivatives accumulate.
void qx_launch_oei(const qx::PairInfo* pairs, int npair, const qx::PrimPair* prims, const double* boys,
                   const double* xyz, const double* Z, int natom, long long n, double* S, double* T, double* V,
                   double* dS, double* dT, double* dV, cudaStream_t s) {
    qx::OeiArgs a;
    a.pairs = pairs;
    a.npair = npair;
    a.prims = prims;
    a.boys = boys;
    a.xyz = xyz;
    a.Z = Z;
    a.natom = natom;
    a.n = n;
    a.S = S;
    a.T = T;
    a.V = V;
    a.dS = dS;
    a.dT = dT;
    a.dV = dV;
    const int blocks = (npair + 3) / 4;
    if (blocks) qx::k_oei<<<blocks, 128, 0, s>>>(a);
}
