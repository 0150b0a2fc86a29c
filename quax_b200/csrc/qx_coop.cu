// qx_coop.cu -- cooperative, table-driven engine for the large angular-momentum
// classes.
//
// One block of COOP_WPB warps owns one contracted shell quartet.  Warp w takes the
// primitive quartets t = w, w+WPB, ... and evaluates the class's VRR program level
// by level: nodes of one level are independent, so lane l evaluates nodes
// l, l+32, ... (four at a time, loads before stores); intermediates live in the
// warp's shared-memory slot array, whose slots the generator recycles by liveness.
// Targets are summed into the warp's accumulators.  The block then adds the warps'
// accumulators and runs the HRR program on them with all its threads, and the
// outputs go through the same epilogues as the straight-line kernels (dense n^4
// scatter, unique blocks, Schwarz diagonal).  Per-thread state stays small, which
// the straight-line per-thread code cannot achieve for (dp|dp) and above.
#include "qx_coop.cuh"
#include "gen/coop_tables.cuh"

#include <algorithm>

namespace qx {

struct CoopArgs {
    EriArgs e;
    CoopClass c;
    int slots;  // doubles of the VRR/HRR buffer region of a block
};

constexpr int COOP_WPB = 4;  // warps per block (one quartet per block)

__device__ __forceinline__ void run_hrr_level(const uint2* __restrict__ hn, int beg, int end, int t, int nthr,
                                              double* V, const double* geo) {
    for (int n0 = beg + t; n0 < end; n0 += nthr * COOP_UNROLL) {
        uint2 d[COOP_UNROLL];
        double r[COOP_UNROLL];
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u)
            if (n0 + u * nthr < end) d[u] = __ldg(hn + n0 + u * nthr);
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u)
            if (n0 + u * nthr < end)
                r[u] = fma(geo[3 * ((d[u].y >> 16) & 1) + ((d[u].y >> 17) & 3)], V[d[u].y & 0xffff], V[d[u].x >> 16]);
#pragma unroll
        for (int u = 0; u < COOP_UNROLL; ++u)
            if (n0 + u * nthr < end) V[d[u].x & 0xffff] = r[u];
    }
}

// One block of COOP_WPB warps per quartet.  Warp w runs primitive quartets
// t = w, w+WPB, ... through the VRR (level by level, lanes in parallel) into its
// own accumulators; the block then sums the warps' accumulators and runs the HRR
// with all its threads.
__global__ void __launch_bounds__(COOP_WPB * 32) k_coop(CoopArgs ca, int mode) {
    const EriArgs& a = ca.e;
    const CoopClass& C = ca.c;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    constexpr int NT = COOP_WPB * 32;
    extern __shared__ double coop_sm[];
    // layout: [COOP_WPB x vslots] VRR buffers (HRR buffer overlays them) |
    //         [COOP_WPB x nacc] accumulators | [COOP_WPB x 24] coefficients
    const int vreg = ca.slots;  // >= max(COOP_WPB * vslots, hslots)
    double* V = coop_sm + (size_t)warp * C.vslots;
    double* accw = coop_sm + vreg + (size_t)warp * C.nacc;
    double* coef = coop_sm + vreg + (size_t)COOP_WPB * C.nacc + warp * 24;
    const long long qi = blockIdx.x;
    if (qi >= a.nq) return;
    const int2 pq = a.quartets[qi];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    if (mode == MODE_JK && jk_screened(a, pq, P, Q)) return;  // whole block, before any barrier
    const uint4* __restrict__ vn = g_coop_vnodes + C.vnode_off;
    const int* __restrict__ vl = g_coop_vlev + C.vlev_off;
    const unsigned short* __restrict__ tg = g_coop_targets + C.tgt_off;
    for (int t = lane; t < C.nacc; t += 32) accw[t] = 0.0;
    const int nk = Q.nprim, ntot = P.nprim * nk;
    for (int t = warp; t < ntot; t += COOP_WPB) {
        const int i = t / nk, j = t - i * nk;
        const PrimPair p = a.prims[P.prim_off + i];
        const PrimPair r = a.prims[Q.prim_off + j];
        __syncwarp();
        coop_prim_setup(p, r, C.S, lane, a.boys, V, coef);
        __syncwarp();
        for (int L = 0; L < C.nvlev; ++L) {
            run_vrr_level(vn, vl[L], vl[L + 1], lane, 32, V, coef);
            __syncwarp();
        }
        for (int t2 = lane; t2 < C.nacc; t2 += 32) accw[t2] += V[tg[t2]];
    }
    __syncthreads();
    // sum the warps' accumulators into the HRR leaves (slots 0..nacc-1)
    double* H = coop_sm;
    double* acc0 = coop_sm + vreg;
    for (int t = tid; t < C.nacc; t += NT) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < COOP_WPB; ++w) s += acc0[(size_t)w * C.nacc + t];
        acc0[t] = s;
    }
    __syncthreads();
    for (int t = tid; t < C.nacc; t += NT) H[t] = acc0[t];
    double* geo = coop_sm + vreg + (size_t)COOP_WPB * C.nacc;  // warp 0's coefficient area
    __syncthreads();
    if (tid == 0) {
        geo[0] = P.ABx; geo[1] = P.ABy; geo[2] = P.ABz;
        geo[3] = Q.ABx; geo[4] = Q.ABy; geo[5] = Q.ABz;
    }
    __syncthreads();
    const uint2* __restrict__ hn = g_coop_hnodes + C.hnode_off;
    const int* __restrict__ hl = g_coop_hlev + C.hlev_off;
    for (int L = 0; L < C.nhlev; ++L) {
        run_hrr_level(hn, hl[L], hl[L + 1], tid, NT, H, geo);
        __syncthreads();
    }
    const unsigned short* __restrict__ outs = g_coop_outs + C.out_off;
    const int NB = (C.lb + 1) * (C.lb + 2) / 2, NC = (C.lc + 1) * (C.lc + 2) / 2, ND = (C.ld + 1) * (C.ld + 2) / 2;
    if (mode == MODE_UNIQUE) {
        for (int o = tid; o < C.nout; o += NT) a.out[a.base + (long long)o * a.nq + qi] = H[outs[o]];
    } else if (mode == MODE_SCHWARZ) {
        double mx = 0.0;
        for (int o = tid; o < C.nout; o += NT) {
            const int ab = o / (NC * ND), cd = o % (NC * ND);
            if (ab == cd) mx = fmax(mx, fabs(H[outs[o]]));
        }
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        __syncthreads();
        if (lane == 0) acc0[warp] = mx;
        __syncthreads();
        if (tid == 0) {
            double m = acc0[0];
            for (int w = 1; w < COOP_WPB; ++w) m = fmax(m, acc0[w]);
            a.out[pq.x] = m;
        }
    } else if (mode == MODE_JK) {
        const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
        for (int o = tid; o < C.nout; o += NT) {
            const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
            jk_images(a.out, a.out2, a.dens, a.n, P.bf1 + ia, P.bf2 + ib, Q.bf1 + ic, Q.bf2 + id, s12, s34, sPQ,
                      H[outs[o]]);
        }
    } else {
        const long long n = a.n;
        const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
        double* __restrict__ out = a.out;
        for (int o = tid; o < C.nout; o += NT) {
            const double v = H[outs[o]];
            const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
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

}  // namespace qx

// Launcher used by the host for classes flagged cooperative (QX_CLASS_COOP).
int qx_coop_index(int cls) {
    for (int i = 0; i < QX_NUM_COOP; ++i)
        if (g_coop_classes[i].cid == cls) return i;
    return -1;
}

void qx_launch_coop(int coop_idx, const qx::EriArgs& a, int mode, cudaStream_t s) {
    using namespace qx;
    const CoopClass& C = g_coop_classes[coop_idx];
    CoopArgs ca;
    ca.e = a;
    ca.c = C;
    const int vreg = std::max(COOP_WPB * C.vslots, C.hslots);
    ca.slots = vreg;
    const size_t smem = sizeof(double) * ((size_t)vreg + (size_t)COOP_WPB * (C.nacc + 24));
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (a.nq) k_coop<<<(unsigned)a.nq, COOP_WPB * 32, smem, s>>>(ca, mode);
}
