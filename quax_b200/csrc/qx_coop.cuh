// qx_coop.cuh -- pieces shared by the cooperative engines (ERI and first
// derivatives): per-order Boys evaluation and one level of a VRR program.
#pragma once
#include "qx_kernels.cuh"

namespace qx {

// F_m(T) for one order m directly from the Taylor table (lane-parallel over m).
__device__ __forceinline__ double boys_one(int m, double T, const double* __restrict__ tab) {
    if (T < BOYS_TMAX) {
        const int g = __double2int_rn(T * BOYS_INV_H);
        const double d = g * (1.0 / BOYS_INV_H) - T;
        const double* row = tab + g * BOYS_NM + m;
        double f = __ldg(row + 7);
#pragma unroll
        for (int k = 6; k >= 0; --k) f = fma(f, d * (1.0 / (k + 1)), __ldg(row + k));
        return f;
    }
    const double rT = 1.0 / T;
    double f = 0.886226925452758013649 * sqrt(rT);
    for (int k = 0; k < m; ++k) f *= (k + 0.5) * rT;
    return f;
}

constexpr int COOP_UNROLL = 4;  // nodes per lane with all loads issued before any store

// Evaluate VRR nodes [beg, end) with `nthr` threads (thread index `t`).
__device__ __forceinline__ void run_vrr_level(const uint4* __restrict__ vn, int beg, int end, int t, int nthr,
                                              double* V, const double* coef) {
    for (int n0 = beg + t; n0 < end; n0 += nthr * COOP_UNROLL) {
        uint4 d[COOP_UNROLL];
        double r[COOP_UNROLL];
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u)
            if (n0 + u * nthr < end) d[u] = __ldg(vn + n0 + u * nthr);
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u) {
            if (n0 + u * nthr < end) {
                const int side = d[u].w & 1, dir = (d[u].w >> 1) & 3;
                const double k = (double)((d[u].w >> 3) & 31), ne = (double)((d[u].w >> 8) & 31);
                const double c1 = coef[6 * side + dir], c2 = coef[6 * side + 3 + dir];
                const double half = coef[12 + 2 * side], ro = coef[13 + 2 * side];
                double v = c1 * V[d[u].x >> 16] + c2 * V[d[u].y & 0xffff];
                v = fma(k * half, V[d[u].y >> 16] - ro * V[d[u].z & 0xffff], v);
                r[u] = fma(ne * coef[16], V[d[u].z >> 16], v);
            }
        }
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u)
            if (n0 + u * nthr < end) V[d[u].x & 0xffff] = r[u];
    }
}


// Scalars of one primitive quartet for the table-driven VRR, written to coef[0..16]:
// PA, WP, QC, WQ, 1/(2 zeta), rho/zeta, 1/(2 eta), rho/eta, 1/(2(zeta+eta)); the
// leaves V[0..S] = pref * F_m and V[S+1] = 0.  Lanes m <= S+1 and lane 31 write.
__device__ __forceinline__ void coop_prim_setup(const PrimPair& p, const PrimPair& r, int S, int lane,
                                                const double* __restrict__ boys, double* V, double* coef) {
    const double ze = p.zeta + r.zeta;
    const double rs = rsqrt(ze);
    const double rze = rs * rs;
    const double PQx = p.Px - r.Px, PQy = p.Py - r.Py, PQz = p.Pz - r.Pz;
    const double T = p.zeta * r.zeta * rze * (PQx * PQx + PQy * PQy + PQz * PQz);
    const double er = r.zeta * rze, pr = p.zeta * rze;
    if (lane <= S) V[lane] = p.K * r.K * rs * boys_one(lane, T, boys);
    if (lane == S + 1) V[lane] = 0.0;
    if (lane == 31) {
        coef[0] = p.PAx; coef[1] = p.PAy; coef[2] = p.PAz;
        coef[3] = -er * PQx; coef[4] = -er * PQy; coef[5] = -er * PQz;
        coef[6] = r.PAx; coef[7] = r.PAy; coef[8] = r.PAz;
        coef[9] = pr * PQx; coef[10] = pr * PQy; coef[11] = pr * PQz;
        coef[12] = p.oo2z; coef[13] = er; coef[14] = r.oo2z; coef[15] = pr; coef[16] = 0.5 * rze;
    }
}

}  // namespace qx
