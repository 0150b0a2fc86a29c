// qx_kernels.cuh -- quartet kernel templates (instantiated one class per
// translation unit in gen/k_eri_<class>.cu so the classes compile in parallel).
#pragma once
#include "qx_device.cuh"
#include "gen/eri_classes.cuh"

namespace qx {

__host__ __device__ constexpr int ncart_h(int l) { return (l + 1) * (l + 2) / 2; }

// ------------------------------------------------------------------ kernels ---
enum { MODE_DENSE = 0, MODE_UNIQUE = 1, MODE_SCHWARZ = 2 };

struct EriArgs {
    const int2* quartets;
    long long nq;
    const PairInfo* pairs;
    const PrimPair* prims;
    const double* boys;
    double* out;
    long long n;     // MODE_DENSE: number of basis functions
    long long base;  // MODE_UNIQUE: offset of this class block
    int* err;
};

template <int LA, int LB, int LC, int LD, int MODE>
__global__ void __launch_bounds__(128) k_eri(EriArgs a) {
    using C = EriCls<LA, LB, LC, LD>;
    const long long qi = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= a.nq) return;
    const int2 pq = a.quartets[qi];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    double acc[C::NACC];
#pragma unroll
    for (int k = 0; k < C::NACC; ++k) acc[k] = 0.0;
    for (int i = 0; i < P.nprim; ++i) {
        const PrimPair p = a.prims[P.prim_off + i];
        for (int j = 0; j < Q.nprim; ++j) {
            const PrimPair r = a.prims[Q.prim_off + j];
            PrimQ q;
            double Fp[C::S + 1];
            prim_setup<C::S>(p, r, a.boys, q, Fp);
            C::vrr(acc, Fp, q);
        }
    }
    double o[C::NOUT];
    C::hrr(acc, o, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz);
    constexpr int NA = ncart_h(LA), NB = ncart_h(LB), NC = ncart_h(LC), ND = ncart_h(LD);
    if constexpr (MODE == MODE_UNIQUE) {
#pragma unroll
        for (int k = 0; k < C::NOUT; ++k) a.out[a.base + (long long)k * a.nq + qi] = o[k];
    } else if constexpr (MODE == MODE_SCHWARZ) {
        double mx = 0.0;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) mx = fmax(mx, fabs(o[((ia * NB + ib) * NC + ia) * ND + ib]));
        a.out[pq.x] = mx;
    } else {
        const long long n = a.n;
        const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
        double* __restrict__ out = a.out;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                    for (int id = 0; id < ND; ++id) {
                        const double v = o[((ia * NB + ib) * NC + ic) * ND + id];
                        const long long i = P.bf1 + ia, j = P.bf2 + ib, k = Q.bf1 + ic, l = Q.bf2 + id;
                        out[((i * n + j) * n + k) * n + l] = v;
                        if (s12) out[((j * n + i) * n + k) * n + l] = v;
                        if (s34) out[((i * n + j) * n + l) * n + k] = v;
                        if (s12 && s34) out[((j * n + i) * n + l) * n + k] = v;
                        if (sPQ) {
                            out[((k * n + l) * n + i) * n + j] = v;
                            if (s34) out[((l * n + k) * n + i) * n + j] = v;
                            if (s12) out[((k * n + l) * n + j) * n + i] = v;
                            if (s12 && s34) out[((l * n + k) * n + j) * n + i] = v;
                        }
                    }
    }
}


template <int LA, int LB, int LC, int LD>
void launch_eri(const EriArgs& a, int mode, cudaStream_t s) {
    const int bs = 128;
    const long long nb = (a.nq + bs - 1) / bs;
    if (nb == 0) return;
    if (mode == MODE_DENSE) k_eri<LA, LB, LC, LD, MODE_DENSE><<<(unsigned)nb, bs, 0, s>>>(a);
    else if (mode == MODE_UNIQUE) k_eri<LA, LB, LC, LD, MODE_UNIQUE><<<(unsigned)nb, bs, 0, s>>>(a);
    else if constexpr (LA == LC && LB == LD) k_eri<LA, LB, LC, LD, MODE_SCHWARZ><<<(unsigned)nb, bs, 0, s>>>(a);
}

typedef void (*EriLaunch)(const EriArgs&, int mode, cudaStream_t);

}  // namespace qx

// one launcher per class, defined in gen/k_eri_<id>.cu
#define QX_DECLARE_LAUNCH(id, a, b, c, d) void qx_launch_eri_##id(const qx::EriArgs&, int, cudaStream_t);
QX_FOR_EACH_CLASS(QX_DECLARE_LAUNCH)
#define QX_DEFINE_LAUNCH(id, a, b, c, d) \
    void qx_launch_eri_##id(const qx::EriArgs& x, int m, cudaStream_t s) { qx::launch_eri<a, b, c, d>(x, m, s); }


