// qx_device.cuh -- device-side data layout, Boys function and quartet kernels.
//
// Layout in HBM (built once per handle by qx_initialize):
//   PrimPair[]  one 80-byte record per primitive pair of every shell pair:
//               zeta, 1/(2 zeta), P, PA = P - A, K = c_a c_b sqrt(2) pi^{5/4}
//               exp(-ab/zeta |AB|^2) / zeta, alpha (for derivative weights).
//   PairInfo[]  one record per shell pair (canonical order: higher AM first):
//               A, AB = A - B, primitive range, basis-function offsets, atoms.
//   int2[]      per angular-momentum class, the screened unique quartets
//               (bra pair, ket pair), sorted by (bra nprim, ket nprim) so the
//               primitive loops of a warp have equal trip counts.
//   double[]    Boys table F_m(T_g), T_g = g/16, g = 0..BOYS_NG-1, m = 0..BOYS_NM-1,
//               row-major [g][m] so the 8 Taylor coefficients of one T are adjacent.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qx {

constexpr int BOYS_NG = 641;        // T in [0, 40]
constexpr int BOYS_NM = 32;         // orders stored
constexpr double BOYS_INV_H = 16.0; // grid spacing 1/16
constexpr double BOYS_TMAX = 40.0;  // above: asymptotic form (e^{-T} < 5e-18)
constexpr int BOYS_TAYLOR = 8;      // Taylor terms k = 0..7

struct __align__(16) PrimPair {
    double zeta, oo2z;
    double Px, Py, Pz;
    double PAx, PAy, PAz;
    double K;
    double alpha;
};

struct __align__(16) PairInfo {
    double Ax, Ay, Az;
    double ABx, ABy, ABz;
    int prim_off, nprim;
    int bf1, bf2;  // first basis function of the canonical first / second shell
    int s1, s2;    // shell indices (canonical order)
    int atom1, atom2;
    int l1, l2;
};

// Per-primitive-quartet scalars consumed by the generated VRR.
template <class T>
struct PrimQT {
    T PAx, PAy, PAz, WPx, WPy, WPz;
    T QCx, QCy, QCz, WQx, WQy, WQz;
    T oo2z, roz, oo2e, roe, oo2ze;
};
using PrimQ = PrimQT<double>;

// FP32 copy of the VRR scalars (mixed precision: the set-up and the Boys
// function stay FP64, the recurrences run in FP32).
__device__ __forceinline__ PrimQT<float> qx_to_float(const PrimQ& q) {
    PrimQT<float> r;
    r.PAx = (float)q.PAx; r.PAy = (float)q.PAy; r.PAz = (float)q.PAz;
    r.WPx = (float)q.WPx; r.WPy = (float)q.WPy; r.WPz = (float)q.WPz;
    r.QCx = (float)q.QCx; r.QCy = (float)q.QCy; r.QCz = (float)q.QCz;
    r.WQx = (float)q.WQx; r.WQy = (float)q.WQy; r.WQz = (float)q.WQz;
    r.oo2z = (float)q.oo2z; r.roz = (float)q.roz; r.oo2e = (float)q.oo2e;
    r.roe = (float)q.roe; r.oo2ze = (float)q.oo2ze;
    return r;
}

// Boys function F_0..F_S(T): 8-term Taylor expansion of the top order about the
// nearest grid point (dF_m/dT = -F_{m+1}), then downward recursion
// F_m = (2T F_{m+1} + e^{-T}) / (2m+1), which is stable.  For T >= 40 the
// asymptotic form F_0 = sqrt(pi/T)/2 with upward recursion F_{m+1} = (2m+1)/(2T) F_m.
// (Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory, sec. 9.8.)
template <int S>
__device__ __forceinline__ void boys(double T, const double* __restrict__ tab, double* F) {
    static_assert(S + BOYS_TAYLOR <= BOYS_NM, "Boys table too short");
    if (T < BOYS_TMAX) {
        const int g = __double2int_rn(T * BOYS_INV_H);
        const double d = g * (1.0 / BOYS_INV_H) - T;
        const double* row = tab + g * BOYS_NM + S;
        double f = __ldg(row + 7);
#pragma unroll
        for (int k = 6; k >= 0; --k) f = fma(f, d * (1.0 / (k + 1)), __ldg(row + k));
        F[S] = f;
        if (S > 0) {
            const double e = exp(-T);
            const double t2 = 2.0 * T;
#pragma unroll
            for (int m = S - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * (1.0 / (2 * m + 1));
        }
    } else {
        const double rT = 1.0 / T;
        F[0] = 0.886226925452758013649 * sqrt(rT);  // sqrt(pi)/2
#pragma unroll
        for (int m = 0; m < S; ++m) F[m + 1] = F[m] * ((m + 0.5) * rT);
    }
}

// Fill the VRR scalars and pref*F_m for one primitive quartet.
template <int S>
__device__ __forceinline__ void prim_setup(const PrimPair& p, const PrimPair& r, const double* __restrict__ boys_tab,
                                           PrimQ& q, double* Fp) {
    const double ze = p.zeta + r.zeta;
    const double rs = rsqrt(ze);
    const double rze = rs * rs;
    const double PQx = p.Px - r.Px, PQy = p.Py - r.Py, PQz = p.Pz - r.Pz;
    const double rho = p.zeta * r.zeta * rze;
    const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
    const double er = r.zeta * rze, pr = p.zeta * rze;
    q.PAx = p.PAx; q.PAy = p.PAy; q.PAz = p.PAz;
    q.QCx = r.PAx; q.QCy = r.PAy; q.QCz = r.PAz;
    q.WPx = -er * PQx; q.WPy = -er * PQy; q.WPz = -er * PQz;
    q.WQx = pr * PQx; q.WQy = pr * PQy; q.WQz = pr * PQz;
    q.oo2z = p.oo2z; q.oo2e = r.oo2z;
    q.roz = er; q.roe = pr; q.oo2ze = 0.5 * rze;
    double F[S + 1];
    boys<S>(T, boys_tab, F);
    const double pref = p.K * r.K * rs;
#pragma unroll
    for (int m = 0; m <= S; ++m) Fp[m] = pref * F[m];
}

}  // namespace qx
