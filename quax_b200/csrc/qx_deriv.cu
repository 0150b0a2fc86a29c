// qx_deriv.cu -- first nuclear derivatives of the ERIs on the cooperative engine.
//
// One block of W warps owns one screened unique quartet.  Warps split the
// primitive quartets; each runs the class's derivative VRR program (one order
// above the plain class) and accumulates four sets: U = sum [e0|f0], WA = sum
// 2 alpha [e0|f0], WB = sum 2 beta [e0|f0], WC = sum 2 gamma [e0|f0].  The block
// sums the warps' sets and runs the derivative HRR program, whose output nodes are
// the nine blocks dA_xyz, dB_xyz, dC_xyz of the Gaussian derivative identity
// d/dA_i g_a = 2 alpha g_{a+1_i} - a_i g_{a-1_i}; dD = -(dA + dB + dC) by
// translational invariance.  Each output node runs its epilogue as soon as it is
// evaluated (outputs are not kept to the end):
//   MODE_DER_DENSE  adds into the reference tensor (3N, n, n, n, n)
//                   (quax/integrals/libint_interface.cc:2582-2779): +d into slice
//                   (atom_c, i), -d into slice (atom_D, i), all 8 images;
//   MODE_DER_SLICE  the same for one nuclear index (compute_2e_deriv with a
//                   one-hot deriv_vec, libint_interface.cc:1097-1335);
//   MODE_GRAD       the adjoint: g[atom, i] += Gamma_sym(abcd) * d, with
//                   Gamma_ijkl = cj D_ij D_kl + ck D_ik D_jl summed over the
//                   quartet's distinct permutational images, so the 3N x n^4
//                   derivative tensor is never formed.
// Quartets whose four shells sit on one atom are skipped, as the reference does.
#include <algorithm>

#include "qx_coop.cuh"
#include "gen/der_tables.cuh"

namespace qx {

enum { MODE_DER_DENSE = 10, MODE_DER_SLICE = 11, MODE_GRAD = 12 };

struct DerArgs {
    EriArgs e;
    DerClass c;
    int W;       // warps per block
    int region;  // doubles of the VRR/HRR buffer region
    const double* D;
    double cj, ck;
    double* grad;  // MODE_GRAD: 3N
    int slice;     // MODE_DER_SLICE: nuclear index
    // split mode: accumulators were summed into acc_in[qi * nacc + t] by k_der_vrr,
    // so k_der only runs the HRR and the epilogue
    const double* acc_in;
};

// One task per warp: (quartet, first primitive quartet) of a fixed chunk; the warp
// runs the VRR over the chunk into shared-memory accumulators and adds them to the
// quartet's global accumulators.  Used for the largest classes, where one quartet's
// primitive loop is too long for a single block to carry the class alone.
constexpr int DER_CHUNK = 64;

__global__ void __launch_bounds__(32) k_der_vrr(DerArgs da, const int2* __restrict__ tasks, long long ntask,
                                                double* __restrict__ acc_out) {
    const EriArgs& a = da.e;
    const DerClass& C = da.c;
    const int lane = threadIdx.x & 31;
    const long long ti = blockIdx.x;
    if (ti >= ntask) return;
    extern __shared__ double dv_sm[];
    double* V = dv_sm;
    double* accw = dv_sm + C.vslots;
    double* coef = accw + C.nacc;
    const int2 task = tasks[ti];
    const int2 pq = a.quartets[task.x];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    const uint4* __restrict__ vn = g_der_vnodes + C.vnode_off;
    const int* __restrict__ vl = g_der_vlev + C.vlev_off;
    const unsigned short* __restrict__ tg = g_der_targets + C.tgt_off;
    const int e1 = C.nu, e2 = C.nu + C.na, e3 = C.nu + C.na + C.nb;
    for (int t = lane; t < C.nacc; t += 32) accw[t] = 0.0;
    const int nk = Q.nprim, ntot = P.nprim * nk;
    const int tend = min(ntot, task.y + DER_CHUNK);
    for (int t = task.y; t < tend; ++t) {
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
        const double w2a = 2.0 * p.alpha, w2b = 2.0 * (p.zeta - p.alpha), w2c = 2.0 * r.alpha;
        for (int t2 = lane; t2 < C.nacc; t2 += 32) {
            const double w = t2 < e1 ? 1.0 : (t2 < e2 ? w2a : (t2 < e3 ? w2b : w2c));
            accw[t2] = fma(w, V[tg[t2]], accw[t2]);
        }
    }
    __syncwarp();
    double* dst = acc_out + (size_t)task.x * C.nacc;
    for (int t = lane; t < C.nacc; t += 32) atomicAdd(dst + t, accw[t]);
}

__device__ __forceinline__ void atomic_images(double* __restrict__ out, long long n, long long i, long long j,
                                              long long k, long long l, bool s12, bool s34, bool sPQ, double v) {
    atomicAdd(out + ((i * n + j) * n + k) * n + l, v);
    if (s12) atomicAdd(out + ((j * n + i) * n + k) * n + l, v);
    if (s34) atomicAdd(out + ((i * n + j) * n + l) * n + k, v);
    if (s12 && s34) atomicAdd(out + ((j * n + i) * n + l) * n + k, v);
    if (sPQ) {
        atomicAdd(out + ((k * n + l) * n + i) * n + j, v);
        if (s34) atomicAdd(out + ((l * n + k) * n + i) * n + j, v);
        if (s12) atomicAdd(out + ((k * n + l) * n + j) * n + i, v);
        if (s12 && s34) atomicAdd(out + ((l * n + k) * n + j) * n + i, v);
    }
}

__global__ void __launch_bounds__(128) k_der(DerArgs da, int mode) {
    const EriArgs& a = da.e;
    const DerClass& C = da.c;
    const int W = da.W, NT = W * 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    extern __shared__ double der_sm[];
    double* V = der_sm + (size_t)warp * C.vslots;
    double* accw = der_sm + da.region + (size_t)warp * C.nacc;
    double* coef = der_sm + da.region + (size_t)W * C.nacc + warp * 24;
    double* gam = der_sm + da.region + (size_t)W * (C.nacc + 24);  // MODE_GRAD: nout weights
    const long long qi = blockIdx.x;
    const int2 pq = a.quartets[qi];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    const int atA = P.atom1, atB = P.atom2, atC = Q.atom1, atD = Q.atom2;
    if (atA == atB && atA == atC && atA == atD) return;  // whole block
    if (mode == MODE_DER_SLICE) {
        const int sa = da.slice / 3;
        if (atA != sa && atB != sa && atC != sa && atD != sa) return;
    }
    const uint4* __restrict__ vn = g_der_vnodes + C.vnode_off;
    const int* __restrict__ vl = g_der_vlev + C.vlev_off;
    const unsigned short* __restrict__ tg = g_der_targets + C.tgt_off;
    const int e1 = C.nu, e2 = C.nu + C.na, e3 = C.nu + C.na + C.nb;
    for (int t = lane; t < C.nacc; t += 32) accw[t] = 0.0;
    const int nk = Q.nprim, ntot = da.acc_in ? 0 : P.nprim * nk;
    for (int t = warp; t < ntot; t += W) {
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
        const double w2a = 2.0 * p.alpha, w2b = 2.0 * (p.zeta - p.alpha), w2c = 2.0 * r.alpha;
        for (int t2 = lane; t2 < C.nacc; t2 += 32) {
            const double w = t2 < e1 ? 1.0 : (t2 < e2 ? w2a : (t2 < e3 ? w2b : w2c));
            accw[t2] = fma(w, V[tg[t2]], accw[t2]);
        }
    }
    __syncthreads();
    double* H = der_sm;
    double* acc0 = der_sm + da.region;
    for (int t = tid; t < C.nacc; t += NT) {
        double s = 0.0;
        if (da.acc_in) {
            s = da.acc_in[(size_t)qi * C.nacc + t];
        } else {
            for (int w = 0; w < W; ++w) s += acc0[(size_t)w * C.nacc + t];
        }
        H[t] = s;
    }
    const int NB = (C.lb + 1) * (C.lb + 2) / 2, NC = (C.lc + 1) * (C.lc + 2) / 2, ND = (C.ld + 1) * (C.ld + 2) / 2;
    const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
    if (mode == MODE_GRAD) {
        const long long n = a.n;
        const double* __restrict__ Dm = da.D;
        const double fJ = (1.0 + sPQ) * (1.0 + s12) * (1.0 + s34), fK = 1.0 + sPQ;
        const double kd = 1.0 + (double)(s12 && s34), kx = (double)s12 + (double)s34;
        for (int o = tid; o < C.nout; o += NT) {
            const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
            const long long i = P.bf1 + ia, j = P.bf2 + ib, k = Q.bf1 + ic, l = Q.bf2 + id;
            const double Dij = __ldg(Dm + i * n + j), Dkl = __ldg(Dm + k * n + l);
            const double Dik = __ldg(Dm + i * n + k), Djl = __ldg(Dm + j * n + l);
            const double Dil = __ldg(Dm + i * n + l), Djk = __ldg(Dm + j * n + k);
            gam[o] = da.cj * fJ * Dij * Dkl + da.ck * fK * (Dik * Djl * kd + Dil * Djk * kx);
        }
    }
    (void)coef;
    __syncthreads();
    if (tid == 0) {
        double* g0 = der_sm + da.region + (size_t)W * C.nacc;
        g0[0] = P.ABx; g0[1] = P.ABy; g0[2] = P.ABz;
        g0[3] = Q.ABx; g0[4] = Q.ABy; g0[5] = Q.ABz;
        g0[6] = -1.0; g0[7] = -2.0; g0[8] = -3.0; g0[9] = -4.0; g0[10] = 0.0;
    }
    const double* geo = der_sm + da.region + (size_t)W * C.nacc;  // warp 0's coefficient area
    __syncthreads();
    const uint2* __restrict__ hn = g_der_hnodes + C.hnode_off;
    const int* __restrict__ hl = g_der_hlev + C.hlev_off;
    const unsigned short* __restrict__ ho = g_der_outs + C.out_off;
    double g9[9];
#pragma unroll
    for (int b = 0; b < 9; ++b) g9[b] = 0.0;
    const int atoms[3] = {atA, atB, atC};
    const long long n = a.n, n4 = n * n * n * n;
    for (int L = 0; L < C.nhlev; ++L) {
        const int end = hl[L + 1];
        for (int nn = hl[L] + tid; nn < end; nn += NT) {
            const uint2 d = __ldg(hn + nn);
            const int side = (d.y >> 16) & 3, dir = (d.y >> 18) & 3;
            const double g = geo[side < 2 ? 3 * side + dir : (side == 2 ? 6 + dir : 10)];
            const double v = fma(g, H[d.y & 0xffff], H[d.x >> 16]);
            H[d.x & 0xffff] = v;
            const int ob = __ldg(ho + nn);
            if (ob == 0xFFFF) continue;
            const int blk = ob / C.nout, o = ob - blk * C.nout;
            if (mode == MODE_GRAD) {
                const double c = gam[o] * v;
#pragma unroll
                for (int b = 0; b < 9; ++b) g9[b] += (b == blk) ? c : 0.0;
            } else {
                const int cen = blk / 3, xyz = blk - 3 * cen;
                const int atc = atoms[cen];
                if (atc == atD) continue;  // +d and -d land in the same slice
                const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
                const long long i = P.bf1 + ia, j = P.bf2 + ib, k = Q.bf1 + ic, l = Q.bf2 + id;
                const int sp = 3 * atc + xyz, sm = 3 * atD + xyz;
                if (mode == MODE_DER_DENSE) {
                    atomic_images(a.out + (long long)sp * n4, n, i, j, k, l, s12, s34, sPQ, v);
                    atomic_images(a.out + (long long)sm * n4, n, i, j, k, l, s12, s34, sPQ, -v);
                } else {
                    if (sp == da.slice) atomic_images(a.out, n, i, j, k, l, s12, s34, sPQ, v);
                    if (sm == da.slice) atomic_images(a.out, n, i, j, k, l, s12, s34, sPQ, -v);
                }
            }
        }
        __syncthreads();
    }
    if (mode == MODE_GRAD) {
        // block reduction of the nine sums, then 12 atomics into the gradient
#pragma unroll
        for (int b = 0; b < 9; ++b)
            for (int off = 16; off > 0; off >>= 1) g9[b] += __shfl_xor_sync(0xffffffffu, g9[b], off);
        double* red = H;  // HRR buffer is free now
        if (lane == 0)
#pragma unroll
            for (int b = 0; b < 9; ++b) red[warp * 9 + b] = g9[b];
        __syncthreads();
        if (tid == 0) {
            double s[9];
            for (int b = 0; b < 9; ++b) {
                s[b] = 0.0;
                for (int w = 0; w < W; ++w) s[b] += red[w * 9 + b];
            }
            for (int x = 0; x < 3; ++x) {
                atomicAdd(da.grad + 3 * atA + x, s[x]);
                atomicAdd(da.grad + 3 * atB + x, s[3 + x]);
                atomicAdd(da.grad + 3 * atC + x, s[6 + x]);
                atomicAdd(da.grad + 3 * atD + x, -(s[x] + s[3 + x] + s[6 + x]));
            }
        }
    }
}

}  // namespace qx

int qx_der_index(int cls) {
    for (int i = 0; i < QX_NUM_DER; ++i)
        if (g_der_classes[i].cid == cls) return i;
    return -1;
}

// Shared-memory plan of a derivative class: warps per block and bytes.
static void der_plan(const DerClass& C, int& W, int& region, size_t& smem) {
    for (W = 4; W >= 1; W >>= 1) {
        region = std::max(W * C.vslots, C.hslots);
        smem = sizeof(double) * ((size_t)region + (size_t)W * (C.nacc + 24) + C.nout);
        if (smem <= 220 * 1024 || W == 1) break;
    }
}

// HRR-only launches (split mode): four warps, no VRR buffers beyond the HRR's.
static void der_plan_hrr(const DerClass& C, int& W, int& region, size_t& smem) {
    W = 4;
    region = C.hslots;
    smem = sizeof(double) * ((size_t)region + (size_t)W * (C.nacc + 24) + C.nout);
    if (smem > 220 * 1024) {
        W = 1;
        smem = sizeof(double) * ((size_t)region + (size_t)(C.nacc + 24) + C.nout);
    }
}

size_t qx_der_smem(int der_idx) {
    int W, region;
    size_t smem;
    der_plan(g_der_classes[der_idx], W, region, smem);
    return smem;
}

// Split mode for the largest classes: `tasks` (quartet, first primitive quartet)
// chunks run the VRR into `scratch` (nq * nacc doubles, zeroed here), then the
// HRR-and-epilogue kernel reads the sums.
void qx_launch_der_split(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck,
                         double* grad, int slice, const int2* tasks, long long ntask, double* scratch, cudaStream_t s) {
    using namespace qx;
    DerArgs da;
    da.e = a;
    da.c = g_der_classes[der_idx];
    da.D = D;
    da.cj = cj;
    da.ck = ck;
    da.grad = grad;
    da.slice = slice;
    da.acc_in = nullptr;
    if (!a.nq) return;
    cudaMemsetAsync(scratch, 0, sizeof(double) * (size_t)a.nq * da.c.nacc, s);
    const size_t vsm = sizeof(double) * ((size_t)da.c.vslots + da.c.nacc + 24);
    if (vsm > 48 * 1024) cudaFuncSetAttribute(k_der_vrr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm);
    if (ntask) k_der_vrr<<<(unsigned)ntask, 32, vsm, s>>>(da, tasks, ntask, scratch);
    size_t smem;
    der_plan_hrr(da.c, da.W, da.region, smem);
    da.acc_in = scratch;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_der, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_der<<<(unsigned)a.nq, da.W * 32, smem, s>>>(da, mode);
}

// HRR and epilogue from accumulator sums that another kernel produced (the
// warp-program VRR of the largest classes): acc holds nq * nacc doubles in this
// engine's accumulator layout.
void qx_launch_der_hrr(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck,
                       double* grad, int slice, const double* acc, cudaStream_t s) {
    using namespace qx;
    DerArgs da;
    da.e = a;
    da.c = g_der_classes[der_idx];
    da.D = D;
    da.cj = cj;
    da.ck = ck;
    da.grad = grad;
    da.slice = slice;
    da.acc_in = acc;
    if (!a.nq) return;
    size_t smem;
    der_plan_hrr(da.c, da.W, da.region, smem);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_der, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_der<<<(unsigned)a.nq, da.W * 32, smem, s>>>(da, mode);
}

long long qx_der_nacc(int der_idx) { return g_der_classes[der_idx].nacc; }
int qx_der_chunk() { return qx::DER_CHUNK; }

void qx_launch_der(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck, double* grad,
                   int slice, cudaStream_t s) {
    using namespace qx;
    DerArgs da;
    da.e = a;
    da.c = g_der_classes[der_idx];
    da.acc_in = nullptr;
    size_t smem;
    der_plan(da.c, da.W, da.region, smem);
    da.D = D;
    da.cj = cj;
    da.ck = ck;
    da.grad = grad;
    da.slice = slice;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_der, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (a.nq) k_der<<<(unsigned)a.nq, da.W * 32, smem, s>>>(da, mode);
}
