// qx_kernels.cuh -- quartet kernel templates (instantiated one class per
// translation unit in gen/k_eri_<class>.cu so the classes compile in parallel).
#pragma once
#include "qx_device.cuh"
#include "gen/eri_classes.cuh"

namespace qx {

__host__ __device__ constexpr int ncart_h(int l) { return (l + 1) * (l + 2) / 2; }

// ------------------------------------------------------------------ kernels ---
enum { MODE_DENSE = 0, MODE_UNIQUE = 1, MODE_SCHWARZ = 2, MODE_JK = 3 };

struct EriArgs {
    const int2* quartets;
    long long nq;
    const PairInfo* pairs;
    const PrimPair* prims;
    const double* boys;
    double* out;
    long long n;     // MODE_DENSE: number of basis functions
    long long base;  // MODE_UNIQUE: offset of this class block
    double* scratch; // ACC_GLOBAL classes: nq * group * NACC doubles
    double* out2;       // MODE_JK: K (out holds J)
    const double* dens; // MODE_JK: D
    int log2g;       // log2 of the lanes cooperating on one quartet (0..5)
    int* err;
    // mixed precision: quartets [nq64, nq) of the list run their recurrences in
    // FP32 (warp and split engines); the default keeps every quartet FP64
    long long nq64 = 0x7fffffffffffffffLL;
    // density screening of J/K (MODE_JK): a quartet is skipped when
    // sqrt(K_ab) sqrt(K_cd) max(|D| over its six shell-pair blocks) < jk_thr
    const double* jk_kpair = nullptr;  // sqrt(Schwarz K) per pair record
    const double* jk_dmax = nullptr;   // max |D| per pair record
    double jk_thr = 0.0;
    // split-mode VRR kernels: primitive-pair records a warp stages into shared
    // memory with the bulk-copy (TMA) engine, bra and ket together; 0 = read them
    // from global memory
    int prim_stage = 0;
    // polls of the bounded wait on those copies before the kernel reports a
    // timeout through the error word
    int wait_limit = 1 << 22;
};

// True when density screening drops this quartet from J/K.
__device__ __forceinline__ bool jk_screened(const EriArgs& a, int2 pq, const PairInfo& P, const PairInfo& Q) {
    if (!a.jk_dmax) return false;
    auto pidx = [](int s, int t) { return s >= t ? s * (s + 1) / 2 + t : t * (t + 1) / 2 + s; };
    double dm = fmax(__ldg(a.jk_dmax + pq.x), __ldg(a.jk_dmax + pq.y));
    dm = fmax(dm, __ldg(a.jk_dmax + pidx(P.s1, Q.s1)));
    dm = fmax(dm, __ldg(a.jk_dmax + pidx(P.s2, Q.s2)));
    dm = fmax(dm, __ldg(a.jk_dmax + pidx(P.s1, Q.s2)));
    dm = fmax(dm, __ldg(a.jk_dmax + pidx(P.s2, Q.s1)));
    return __ldg(a.jk_kpair + pq.x) * __ldg(a.jk_kpair + pq.y) * dm < a.jk_thr;
}

// Accumulator storage for the contracted [e0|f0] targets of one quartet.
template <int N>
struct RegAcc {
    double v[N];
    __device__ __forceinline__ double& operator()(int k) { return v[k]; }
};
struct StridedAcc {  // shared or global memory, element k of thread t at base[k*stride + t]
    double* base;
    long long stride;
    __device__ __forceinline__ double& operator()(int k) { return base[(long long)k * stride]; }
};

// Accumulator placement per class: registers when small, shared memory (per
// thread, conflict-free SoA) when mid-sized, global scratch when even 32 threads'
// worth does not fit in shared memory.
enum { ACC_REG = 0, ACC_SMEM = 1, ACC_GLOBAL = 2 };
template <int NACC>
struct AccPolicy {
    static constexpr int kind = NACC <= 48 ? ACC_REG : (NACC <= 220 ? ACC_SMEM : ACC_GLOBAL);
    static constexpr int bs = 128;
    static constexpr int smem = kind == ACC_SMEM ? NACC * bs * 8 : 0;
};

// Direct Coulomb/exchange build: every distinct image (p q|r s) of a unique element
// adds v D_rs to J_pq and v D_qs to K_pr (J_ij = sum_kl (ij|kl) D_kl and
// K_ij = sum_kl (ik|jl) D_kl, the reference's jk_build on G and on G.transpose(0,2,1,3)).
__device__ __forceinline__ void jk_image(double* __restrict__ J, double* __restrict__ K,
                                         const double* __restrict__ D, long long n, long long p, long long q,
                                         long long r, long long s, double v) {
    atomicAdd(J + p * n + q, v * __ldg(D + r * n + s));
    atomicAdd(K + p * n + r, v * __ldg(D + q * n + s));
}

__device__ __forceinline__ void jk_images(double* __restrict__ J, double* __restrict__ K, const double* __restrict__ D,
                                          long long n, long long i, long long j, long long k, long long l, bool s12,
                                          bool s34, bool sPQ, double v) {
    jk_image(J, K, D, n, i, j, k, l, v);
    if (s12) jk_image(J, K, D, n, j, i, k, l, v);
    if (s34) jk_image(J, K, D, n, i, j, l, k, v);
    if (s12 && s34) jk_image(J, K, D, n, j, i, l, k, v);
    if (sPQ) {
        jk_image(J, K, D, n, k, l, i, j, v);
        if (s34) jk_image(J, K, D, n, l, k, i, j, v);
        if (s12) jk_image(J, K, D, n, k, l, j, i, v);
        if (s12 && s34) jk_image(J, K, D, n, l, k, j, i, v);
    }
}

template <int NA, int NB, int NC, int ND>
struct JKStore {
    double* __restrict__ J;
    double* __restrict__ K;
    const double* __restrict__ D;
    long long n;
    int bf1, bf2, bf3, bf4;
    bool s12, s34, sPQ;
    __device__ __forceinline__ void operator()(int k, double v) {
        const int id = k % ND, ic = (k / ND) % NC, ib = (k / (ND * NC)) % NB, ia = k / (ND * NC * NB);
        jk_images(J, K, D, n, bf1 + ia, bf2 + ib, bf3 + ic, bf4 + id, s12, s34, sPQ, v);
    }
};

template <int NA, int NB, int NC, int ND>
struct UniqueStore {
    double* out;
    long long base, nq, qi;
    __device__ __forceinline__ void operator()(int k, double v) { out[base + (long long)k * nq + qi] = v; }
};

template <int NA, int NB, int NC, int ND>
struct SchwarzStore {
    double mx = 0.0;
    __device__ __forceinline__ void operator()(int k, double v) {
        const int ab = k / (NC * ND), cd = k % (NC * ND);
        if (ab == cd) mx = fmax(mx, fabs(v));
    }
};

// Writes one element of a unique quartet to all its images in the dense n^4
// tensor (8-fold permutational symmetry, images deduplicated by the flags).
template <int NA, int NB, int NC, int ND>
struct DenseStore {
    double* __restrict__ out;
    long long n;
    int bf1, bf2, bf3, bf4;
    bool s12, s34, sPQ;
    __device__ __forceinline__ void operator()(int k, double v) {
        const int id = k % ND, ic = (k / ND) % NC, ib = (k / (ND * NC)) % NB, ia = k / (ND * NC * NB);
        const long long i = bf1 + ia, j = bf2 + ib, kk = bf3 + ic, l = bf4 + id;
        out[((i * n + j) * n + kk) * n + l] = v;
        if (s12) out[((j * n + i) * n + kk) * n + l] = v;
        if (s34) out[((i * n + j) * n + l) * n + kk] = v;
        if (s12 && s34) out[((j * n + i) * n + l) * n + kk] = v;
        if (sPQ) {
            out[((kk * n + l) * n + i) * n + j] = v;
            if (s34) out[((l * n + kk) * n + i) * n + j] = v;
            if (s12) out[((kk * n + l) * n + j) * n + i] = v;
            if (s12 && s34) out[((l * n + kk) * n + j) * n + i] = v;
        }
    }
};

// Primitive loop of one contracted quartet.  The G = 2^log2g lanes of a group
// take primitive quartets t = sub, sub+G, ...; afterwards the group's partial
// accumulators are summed with butterfly shuffles into lane sub == 0.
template <class C, class Acc>
__device__ __forceinline__ void contract_quartet(const EriArgs& a, const PairInfo& P, const PairInfo& Q, Acc& acc,
                                                 int sub, bool active) {
#pragma unroll
    for (int k = 0; k < C::NACC; ++k) acc(k) = 0.0;
    const int nk = Q.nprim;
    const int ntot = active ? P.nprim * nk : 0;
    const int G = 1 << a.log2g;
    for (int t = sub; t < ntot; t += G) {
        const int i = t / nk, j = t - i * nk;
        const PrimPair p = a.prims[P.prim_off + i];
        const PrimPair r = a.prims[Q.prim_off + j];
        PrimQ q;
        double Fp[C::S + 1];
        prim_setup<C::S>(p, r, a.boys, q, Fp);
        C::vrr(acc, Fp, q);
    }
    if (a.log2g) {
#pragma unroll 1
        for (int k = 0; k < C::NACC; ++k) {
            double v = acc(k);
            for (int off = G >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            acc(k) = v;
        }
    }
}

template <class C, int LA, int LB, int LC, int LD, int MODE, class Acc>
__device__ __noinline__ void finish_quartet(const EriArgs& a, const PairInfo& P, const PairInfo& Q, int2 pq,
                                            long long qi, Acc acc) {
    constexpr int NA = ncart_h(LA), NB = ncart_h(LB), NC = ncart_h(LC), ND = ncart_h(LD);
    if constexpr (MODE == MODE_UNIQUE) {
        UniqueStore<NA, NB, NC, ND> st{a.out, a.base, a.nq, qi};
        C::hrr(acc, st, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz);
    } else if constexpr (MODE == MODE_SCHWARZ) {
        SchwarzStore<NA, NB, NC, ND> st;
        C::hrr(acc, st, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz);
        a.out[pq.x] = st.mx;
    } else if constexpr (MODE == MODE_JK) {
        JKStore<NA, NB, NC, ND> st{a.out, a.out2, a.dens, a.n, P.bf1, P.bf2, Q.bf1, Q.bf2,
                                   P.s1 != P.s2, Q.s1 != Q.s2, pq.x != pq.y};
        C::hrr(acc, st, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz);
    } else {
        DenseStore<NA, NB, NC, ND> st{a.out, a.n, P.bf1, P.bf2, Q.bf1, Q.bf2, P.s1 != P.s2, Q.s1 != Q.s2, pq.x != pq.y};
        C::hrr(acc, st, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz);
    }
}

template <int LA, int LB, int LC, int LD, int MODE>
__global__ void __launch_bounds__(AccPolicy<EriCls<LA, LB, LC, LD>::NACC>::bs) k_eri(EriArgs a) {
    using C = EriCls<LA, LB, LC, LD>;
    using Pol = AccPolicy<C::NACC>;
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long qi = gt >> a.log2g;
    const int sub = (int)(gt & ((1 << a.log2g) - 1));
    bool active = qi < a.nq;
    // every lane stays to the end: the group reduction shuffles over the full warp
    const int2 pq = active ? a.quartets[qi] : make_int2(0, 0);
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    if (MODE == MODE_JK && active && jk_screened(a, pq, P, Q)) active = false;  // group-uniform
    if constexpr (Pol::kind == ACC_REG) {
        RegAcc<C::NACC> acc;
        contract_quartet<C>(a, P, Q, acc, sub, active);
        if (active && sub == 0) finish_quartet<C, LA, LB, LC, LD, MODE>(a, P, Q, pq, qi, acc);
    } else if constexpr (Pol::kind == ACC_SMEM) {
        extern __shared__ double smem_acc[];
        StridedAcc acc{smem_acc + threadIdx.x, Pol::bs};
        contract_quartet<C>(a, P, Q, acc, sub, active);
        if (active && sub == 0) finish_quartet<C, LA, LB, LC, LD, MODE>(a, P, Q, pq, qi, acc);
    } else {
        const long long nthreads = (long long)gridDim.x * blockDim.x;
        StridedAcc acc{a.scratch + gt, nthreads};
        contract_quartet<C>(a, P, Q, acc, sub, active);
        if (active && sub == 0) finish_quartet<C, LA, LB, LC, LD, MODE>(a, P, Q, pq, qi, acc);
    }
}

template <int LA, int LB, int LC, int LD>
void launch_eri(const EriArgs& a, int mode, cudaStream_t s) {
    using Pol = AccPolicy<EriCls<LA, LB, LC, LD>::NACC>;
    const int bs = Pol::bs;
    const long long nb = ((a.nq << a.log2g) + bs - 1) / bs;
    if (nb == 0) return;
    if (mode == MODE_DENSE) {
        auto k = k_eri<LA, LB, LC, LD, MODE_DENSE>;
        if (Pol::smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, Pol::smem);
        k<<<(unsigned)nb, bs, Pol::smem, s>>>(a);
    } else if (mode == MODE_UNIQUE) {
        auto k = k_eri<LA, LB, LC, LD, MODE_UNIQUE>;
        if (Pol::smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, Pol::smem);
        k<<<(unsigned)nb, bs, Pol::smem, s>>>(a);
    } else if (mode == MODE_JK) {
        auto k = k_eri<LA, LB, LC, LD, MODE_JK>;
        if (Pol::smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, Pol::smem);
        k<<<(unsigned)nb, bs, Pol::smem, s>>>(a);
    } else if constexpr (LA == LC && LB == LD) {
        auto k = k_eri<LA, LB, LC, LD, MODE_SCHWARZ>;
        if (Pol::smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, Pol::smem);
        k<<<(unsigned)nb, bs, Pol::smem, s>>>(a);
    }
}

// Doubles of global scratch a class needs per quartet (0 unless ACC_GLOBAL).
template <int LA, int LB, int LC, int LD>
constexpr long long scratch_per_quartet() {
    using C = EriCls<LA, LB, LC, LD>;
    return AccPolicy<C::NACC>::kind == ACC_GLOBAL ? C::NACC : 0;
}

typedef void (*EriLaunch)(const EriArgs&, int mode, cudaStream_t);

}  // namespace qx

// one launcher per class, defined in gen/k_eri_<id>.cu
#define QX_DECLARE_LAUNCH(id, a, b, c, d) void qx_launch_eri_##id(const qx::EriArgs&, int, cudaStream_t);
QX_FOR_EACH_SL_CLASS(QX_DECLARE_LAUNCH)
int qx_coop_index(int cls);
void qx_launch_coop(int coop_idx, const qx::EriArgs& a, int mode, cudaStream_t s);
#define QX_DEFINE_LAUNCH(id, a, b, c, d) \
    void qx_launch_eri_##id(const qx::EriArgs& x, int m, cudaStream_t s) { qx::launch_eri<a, b, c, d>(x, m, s); }
#define QX_SCRATCH_ENTRY(id, a, b, c, d) qx::scratch_per_quartet<a, b, c, d>(),


