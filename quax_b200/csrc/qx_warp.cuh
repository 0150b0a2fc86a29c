// qx_warp.cuh -- warp-per-quartet kernels: lanes = primitive quartets.
//
// One warp owns one contracted shell quartet.  Its 32 lanes take 32 primitive
// quartets at a time and each runs the class's generated straight-line VRR in
// registers.  Every VRR target (times its weight, for the derivative sets) is an
// "item"; items are staged 16 at a time and folded across the warp with a
// transposing butterfly of shuffles (reduce16: 16 shuffles per 16 items per lane),
// after which lane 2j holds the warp sum of item j and adds it to the warp's
// shared-memory accumulator.  So no lane keeps a full accumulator set -- the
// obstacle for straight-line per-thread code on classes with hundreds of
// targets -- and the per-primitive work stays in registers.  After the primitive
// loop the warp runs the class's table-driven HRR program on the accumulators
// (lanes in parallel, level by level) and the usual epilogues.
#pragma once
#include "qx_kernels.cuh"

namespace qx {

struct WarpArgs {
    EriArgs e;
    int wpq;  // warps per quartet: 1 (a block holds 4 quartets) or 4 (a block holds one)
    const double* D;  // adjoint: density (n x n)
    double cj, ck;
    double* grad;  // adjoint: 3N
    int slice;     // single derivative slice
    const double* dir = nullptr;  // Hessian-vector product: direction (3N)
    // split mode: the quartets' accumulators (NITEM_PAD per quartet, item order)
    // were summed by k_gvrr; the kernel runs only the HRR and the epilogue
    const double* acc_in = nullptr;
    // derivative tile (WMODE_DER_TILE): out is a (3N, tile_E) row-major buffer,
    // element qi * NOUT + o (tile_images = 0), or (qi * NOUT + o) * 8 + image for
    // each distinct image of the integral (tile_images = 1)
    long long tile_E = 0;
    int tile_images = 0;
};

enum { WMODE_DENSE = 0, WMODE_UNIQUE = 1, WMODE_SCHWARZ = 2, WMODE_DER_DENSE = 10, WMODE_DER_SLICE = 11,
       WMODE_GRAD = 12, WMODE_DER2_DENSE = 13, WMODE_DER2_SLICE = 14, WMODE_HVP = 15, WMODE_DER_TILE = 16 };

// Adds v to row `row` of a derivative tile at element e of quartet-local index:
// once (unique elements) or into the slot of every distinct image (8 per element;
// the images (ij|kl), (ji|kl), (ij|lk), (ji|lk), (kl|ij), (lk|ij), (kl|ji), (lk|ji)).
__device__ __forceinline__ void tile_add(double* __restrict__ B, long long E, int row, long long e, bool images,
                                         bool s12, bool s34, bool sPQ, double v) {
    double* r = B + (long long)row * E;
    if (!images) {
        atomicAdd(r + e, v);
        return;
    }
    double* b = r + e * 8;
    atomicAdd(b + 0, v);
    if (s12) atomicAdd(b + 1, v);
    if (s34) atomicAdd(b + 2, v);
    if (s12 && s34) atomicAdd(b + 3, v);
    if (sPQ) {
        atomicAdd(b + 4, v);
        if (s34) atomicAdd(b + 5, v);
        if (s12) atomicAdd(b + 6, v);
        if (s12 && s34) atomicAdd(b + 7, v);
    }
}

constexpr int WARP_QPB = 4;  // quartets (warps) per block

// Sum item k of the 16 staged values over the warp; lane 2j ends with item j
// (in v[0]).
__device__ __forceinline__ void reduce16_core(double (&v)[16], unsigned lane) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const bool up = lane & 16;
        const double send = up ? v[i] : v[i + 8];
        const double keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool up = lane & 8;
        const double send = up ? v[i] : v[i + 4];
        const double keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const bool up = lane & 4;
        const double send = up ? v[i] : v[i + 2];
        const double keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool up = lane & 2;
        const double send = up ? v[0] : v[1];
        const double keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}

__device__ __forceinline__ void reduce16(double (&v)[16], double* __restrict__ acc16, unsigned lane) {
    reduce16_core(v, lane);
    if (!(lane & 1)) acc16[(lane >> 1) & 15] += v[0];
}

// Where a warp program's staged items go: the warp's shared-memory accumulators
// (item order), or a quartet's global accumulators through an item -> slot map
// (atomic adds: several warps share a quartet).
struct SmemSink {
    double* acc;
    __device__ __forceinline__ void operator()(double (&v)[16], int base, unsigned lane) const {
        reduce16(v, acc + base, lane);
    }
};

struct IdentSink {
    double* acc;
    __device__ __forceinline__ void operator()(double (&v)[16], int base, unsigned lane) const {
        reduce16_core(v, lane);
        if (!(lane & 1)) atomicAdd(acc + base + (lane >> 1), v[0]);
    }
};

struct GlobalSink {
    double* acc;
    const unsigned short* map;
    __device__ __forceinline__ void operator()(double (&v)[16], int base, unsigned lane) const {
        reduce16_core(v, lane);
        if (!(lane & 1)) {
            const unsigned m = __ldg(map + base + (lane >> 1));
            if (m != 0xFFFFu) atomicAdd(acc + m, v[0]);
        }
    }
};

// Bulk copies global -> shared memory through the TMA unit (cp.async.bulk, no
// tensor map, no multicast), completed on a shared-memory mbarrier.  The waits are
// bounded: a copy that has not landed after `limit` polls makes the kernel report
// an error word instead of spinning on.
__device__ __forceinline__ unsigned qx_smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void qx_mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(qx_smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void qx_mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(qx_smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void qx_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     qx_smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(qx_smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool qx_mbar_wait(unsigned long long* bar, unsigned phase, int limit) {
    for (int it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(qx_smem_u32(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Chunked warp programs: the lane's VRR inputs are saved once per primitive
// quartet (lane-strided, bank-conflict free) and every later chunk reloads them
// with volatile loads, so the compiler cannot merge a chunk's recomputed
// intermediates with an earlier chunk's and keep them all live.
template <int NF, class T>
__device__ __forceinline__ void qx_save_inputs(const PrimQT<T>& q, const T* Fp, T* save, unsigned lane) {
    T* s = save + lane;
    s[0 * 32] = q.PAx; s[1 * 32] = q.PAy; s[2 * 32] = q.PAz;
    s[3 * 32] = q.WPx; s[4 * 32] = q.WPy; s[5 * 32] = q.WPz;
    s[6 * 32] = q.QCx; s[7 * 32] = q.QCy; s[8 * 32] = q.QCz;
    s[9 * 32] = q.WQx; s[10 * 32] = q.WQy; s[11 * 32] = q.WQz;
    s[12 * 32] = q.oo2z; s[13 * 32] = q.roz; s[14 * 32] = q.oo2e;
    s[15 * 32] = q.roe; s[16 * 32] = q.oo2ze;
#pragma unroll
    for (int m = 0; m < NF; ++m) s[(17 + m) * 32] = Fp[m];
}

template <int NF, class T>
__device__ __forceinline__ void qx_load_inputs(const T* save, unsigned lane, PrimQT<T>& q, T* F) {
    const volatile T* s = save + lane;
    q.PAx = s[0 * 32]; q.PAy = s[1 * 32]; q.PAz = s[2 * 32];
    q.WPx = s[3 * 32]; q.WPy = s[4 * 32]; q.WPz = s[5 * 32];
    q.QCx = s[6 * 32]; q.QCy = s[7 * 32]; q.QCz = s[8 * 32];
    q.WQx = s[9 * 32]; q.WQy = s[10 * 32]; q.WQz = s[11 * 32];
    q.oo2z = s[12 * 32]; q.roz = s[13 * 32]; q.oo2e = s[14 * 32];
    q.roe = s[15 * 32]; q.oo2ze = s[16 * 32];
#pragma unroll
    for (int m = 0; m < NF; ++m) F[m] = s[(17 + m) * 32];
}

// Table-driven HRR level loop for one warp.  Node (uint2): x = dst | s1<<16,
// y = s2 | g<<16 ; V[dst] = V[s1] + geo[g] V[s2] with geo = AB_xyz, CD_xyz, then the
// integer constants -8..7 (linear combinations of shifted blocks in the
// derivative programs).
template <class OnOut>
__device__ __forceinline__ void warp_hrr(const uint2* __restrict__ hn, const int* __restrict__ hl, int nhlev,
                                         const unsigned short* __restrict__ ho, double* H, const double* geo,
                                         unsigned lane, OnOut&& on_out) {
    for (int L = 0; L < nhlev; ++L) {
        const int end = __ldg(hl + L + 1);
        for (int nn = __ldg(hl + L) + lane; nn < end; nn += 32) {
            const uint2 d = __ldg(hn + nn);
            const double v = fma(geo[(d.y >> 16) & 31], H[d.y & 0xffff], H[d.x >> 16]);
            H[d.x & 0xffff] = v;
            if (ho) {
                const int ob = __ldg(ho + nn);
                if (ob != 0xFFFF) on_out(ob, v);
            }
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void dense_images(double* __restrict__ out, long long n, long long i, long long j,
                                             long long k, long long l, bool s12, bool s34, bool sPQ, double v) {
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

__device__ __forceinline__ void atomic_images_w(double* __restrict__ out, long long n, long long i, long long j,
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

// W: generated class (VRR + table offsets); DERIV selects the derivative program.
template <class W, int DERIV>
__global__ void __launch_bounds__(WARP_QPB * 32) k_warp(WarpArgs wa, int mode) {
    const EriArgs& a = wa.e;
    const unsigned lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // wpq = 4: the block's four warps split one quartet's primitive batches
    const int wpq = wa.wpq;
    const int sub = warp % wpq;
    const long long qi = (long long)blockIdx.x * (WARP_QPB / wpq) + warp / wpq;
    if (qi >= a.nq) return;  // whole warp (whole block when wpq = 4)
    extern __shared__ double warp_sm[];
    double* H = warp_sm + (size_t)warp * W::SMEM_PER_WARP;  // accumulators = HRR leaves
    double* geo = H + W::HSLOTS;                             // 6 geometry factors + constants -8..7
    double* gam = geo + 32;                                  // adjoint: Gamma weights (NOUT)
    double* save = H + (W::SMEM_PER_WARP - W::SAVE);         // chunked VRR: saved lane inputs
    const int2 pq = a.quartets[qi];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    const int atA = P.atom1, atB = P.atom2, atC = Q.atom1, atD = Q.atom2;
    const bool f32 = qi >= a.nq64;  // warp-uniform: one quartet per warp
    // density screening (J/K): the whole warp, or all warps of a wpq = 4 block
    if (!DERIV && mode == MODE_JK && jk_screened(a, pq, P, Q)) return;
    if (DERIV) {
        if (atA == atB && atA == atC && atA == atD) return;  // reference skips these
        if (mode == WMODE_DER_SLICE) {
            const int sa = wa.slice / 3;
            if (atA != sa && atB != sa && atC != sa && atD != sa) return;
        }
        if (mode == WMODE_DER2_SLICE) {
            const int s1 = wa.slice & 0xffff, s2 = wa.slice >> 16;  // nuclear indices nu1 <= nu2
            const int a1 = s1 / 3, a2 = s2 / 3;
            if ((atA != a1 && atB != a1 && atC != a1 && atD != a1) || (atA != a2 && atB != a2 && atC != a2 && atD != a2))
                return;
        }
        if (DERIV == 2 && mode == WMODE_HVP) {
            // a quartet whose four atoms move alike along v (w_X = v(X) - v(D) = 0
            // for X = A, B, C) adds nothing: every term is linear in w.  For a
            // Hessian column (v on one atom) that is every quartet off that atom.
            bool still = true;
            for (int x = 0; x < 3; ++x) {
                const double vD = __ldg(wa.dir + 3 * atD + x);
                still = still && __ldg(wa.dir + 3 * atA + x) == vD && __ldg(wa.dir + 3 * atB + x) == vD &&
                        __ldg(wa.dir + 3 * atC + x) == vD;
            }
            if (still) return;  // whole warp (whole block when wpq = 4): one quartet
        }
    }
    if (wa.acc_in) {
        const double* __restrict__ src = wa.acc_in + (size_t)qi * W::NITEM_PAD;
        for (int t = lane; t < W::NITEM_PAD; t += 32) H[t] = src[t];
    } else {
        for (int t = lane; t < W::NITEM_PAD; t += 32) H[t] = 0.0;
    }
    __syncwarp();
    const int nk = Q.nprim, ntot = wa.acc_in ? 0 : P.nprim * nk;
    for (int t0 = 32 * sub; t0 < ntot; t0 += 32 * wpq) {
        const int t = t0 + (int)lane;
        const bool act = t < ntot;
        const int tt = act ? t : 0;
        const int i = tt / nk, j = tt - i * nk;
        const PrimPair p = a.prims[P.prim_off + i];
        const PrimPair r = a.prims[Q.prim_off + j];
        PrimQ q;
        double Fp[W::S + 1];
        prim_setup<W::S>(p, r, a.boys, q, Fp);
        if (!act) {
#pragma unroll
            for (int m = 0; m <= W::S; ++m) Fp[m] = 0.0;
        }
        const double w1 = 2.0 * p.alpha, w2 = 2.0 * (p.zeta - p.alpha), w3 = 2.0 * r.alpha;
        if constexpr (DERIV < 2) {
            if (f32) {
                float Ff[W::S + 1];
#pragma unroll
                for (int m = 0; m <= W::S; ++m) Ff[m] = (float)Fp[m];
                W::vrr(Ff, qx_to_float(q), w1, w2, w3, SmemSink{H}, lane, reinterpret_cast<float*>(save));
            } else {
                W::vrr(Fp, q, w1, w2, w3, SmemSink{H}, lane, save);
            }
        } else {
            W::vrr(Fp, q, w1, w2, w3, SmemSink{H}, lane, save);
        }
        __syncwarp();
    }
    if (wpq > 1) {
        // sum the four warps' accumulators into warp 0's; warp 0 finishes alone
        __syncthreads();
        for (int t = threadIdx.x; t < W::NITEM_PAD; t += 32 * WARP_QPB) {
            double s = 0.0;
#pragma unroll
            for (int w = 1; w < WARP_QPB; ++w) s += warp_sm[(size_t)w * W::SMEM_PER_WARP + t];
            warp_sm[t] += s;
        }
        __syncthreads();
        if (warp != 0) return;
    }
    if (lane == 0) {
        geo[0] = P.ABx; geo[1] = P.ABy; geo[2] = P.ABz;
        geo[3] = Q.ABx; geo[4] = Q.ABy; geo[5] = Q.ABz;
    }
    if (lane < 16) geo[6 + lane] = (double)((int)lane - 8);
    constexpr int NB = ncart_h(W::LB), NC = ncart_h(W::LC), ND = ncart_h(W::LD);
    const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
    const long long n = a.n;
    if ((DERIV == 1 && mode == WMODE_GRAD) || (DERIV == 2 && mode == WMODE_HVP)) {
        const double* __restrict__ Dm = wa.D;
        const double fJ = (1.0 + sPQ) * (1.0 + s12) * (1.0 + s34), fK = 1.0 + sPQ;
        const double kd = 1.0 + (double)(s12 && s34), kx = (double)s12 + (double)s34;
        for (int o = lane; o < W::NOUT; o += 32) {
            const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
            const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
            gam[o] = wa.cj * fJ * __ldg(Dm + ii * n + jj) * __ldg(Dm + kk * n + ll) +
                     wa.ck * fK * (__ldg(Dm + ii * n + kk) * __ldg(Dm + jj * n + ll) * kd +
                                   __ldg(Dm + ii * n + ll) * __ldg(Dm + jj * n + kk) * kx);
        }
    }
    __syncwarp();
    if (!DERIV) {
        warp_hrr(W::hnodes(), W::hlev(), W::NHLEV, nullptr, H, geo, lane, [](int, double) {});
        const unsigned short* __restrict__ outs = W::outs();
        if (mode == WMODE_UNIQUE) {
            for (int o = lane; o < W::NOUT; o += 32) a.out[a.base + (long long)o * a.nq + qi] = H[__ldg(outs + o)];
        } else if (mode == WMODE_SCHWARZ) {
            double mx = 0.0;
            for (int o = lane; o < W::NOUT; o += 32) {
                const int ab = o / (NC * ND), cd = o % (NC * ND);
                if (ab == cd) mx = fmax(mx, fabs(H[__ldg(outs + o)]));
            }
            for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
            if (lane == 0) a.out[pq.x] = mx;
        } else if (mode == MODE_JK) {
            // J/K from the whole quartet block at once: the up-to-8 images of each
            // integral regroup into six block contractions with D (JA = G.D_CD over
            // the ket, JC = D_AB.G over the bra, and the four exchange blocks), so
            // each touched J/K entry takes one atomic per quartet instead of one per
            // integral and image.
            constexpr int NA = ncart_h(W::LA);
            const double* __restrict__ Dm = a.dens;
            double* __restrict__ Jm = a.out;
            double* __restrict__ Km = a.out2;
            const long long bA = P.bf1, bB = P.bf2, bC = Q.bf1, bD = Q.bf2;
            auto G = [&](int ia, int ib, int ic, int id) {
                return H[__ldg(outs + ((ia * NB + ib) * NC + ic) * ND + id)];
            };
            auto Dv = [&](long long r, long long c) { return __ldg(Dm + r * n + c); };
            constexpr int nJA = NA * NB, nJC = NC * ND, nK1 = NA * NC, nK2 = NB * NC, nK3 = NA * ND, nK4 = NB * ND;
            constexpr int total = nJA + nJC + nK1 + nK2 + nK3 + nK4;
            for (int e = lane; e < total; e += 32) {
                int r = e;
                if (r < nJA) {  // J_ij += (1 + s34) sum_kl G D_kl, and J_ji with s12
                    const int ia = r / NB, ib = r % NB;
                    double x = 0.0;
                    for (int ic = 0; ic < NC; ++ic)
                        for (int id = 0; id < ND; ++id) x = fma(G(ia, ib, ic, id), Dv(bC + ic, bD + id), x);
                    x *= 1.0 + s34;
                    atomicAdd(Jm + (bA + ia) * n + bB + ib, x);
                    if (s12) atomicAdd(Jm + (bB + ib) * n + bA + ia, x);
                    continue;
                }
                r -= nJA;
                if (r < nJC) {  // with sPQ: J_kl += (1 + s12) sum_ij G D_ij, and J_lk with s34
                    if (!sPQ) continue;
                    const int ic = r / ND, id = r % ND;
                    double x = 0.0;
                    for (int ia = 0; ia < NA; ++ia)
                        for (int ib = 0; ib < NB; ++ib) x = fma(G(ia, ib, ic, id), Dv(bA + ia, bB + ib), x);
                    x *= 1.0 + s12;
                    atomicAdd(Jm + (bC + ic) * n + bD + id, x);
                    if (s34) atomicAdd(Jm + (bD + id) * n + bC + ic, x);
                    continue;
                }
                r -= nJC;
                if (r < nK1) {  // K_ik += sum_jl G D_jl (and K_ki with sPQ)
                    const int ia = r / NC, ic = r % NC;
                    double x = 0.0;
                    for (int ib = 0; ib < NB; ++ib)
                        for (int id = 0; id < ND; ++id) x = fma(G(ia, ib, ic, id), Dv(bB + ib, bD + id), x);
                    atomicAdd(Km + (bA + ia) * n + bC + ic, x);
                    if (sPQ) atomicAdd(Km + (bC + ic) * n + bA + ia, x);
                    continue;
                }
                r -= nK1;
                if (r < nK2) {  // with s12: K_jk += sum_il G D_il (and K_kj with sPQ)
                    if (!s12) continue;
                    const int ib = r / NC, ic = r % NC;
                    double x = 0.0;
                    for (int ia = 0; ia < NA; ++ia)
                        for (int id = 0; id < ND; ++id) x = fma(G(ia, ib, ic, id), Dv(bA + ia, bD + id), x);
                    atomicAdd(Km + (bB + ib) * n + bC + ic, x);
                    if (sPQ) atomicAdd(Km + (bC + ic) * n + bB + ib, x);
                    continue;
                }
                r -= nK2;
                if (r < nK3) {  // with s34: K_il += sum_jk G D_jk (and K_li with sPQ)
                    if (!s34) continue;
                    const int ia = r / ND, id = r % ND;
                    double x = 0.0;
                    for (int ib = 0; ib < NB; ++ib)
                        for (int ic = 0; ic < NC; ++ic) x = fma(G(ia, ib, ic, id), Dv(bB + ib, bC + ic), x);
                    atomicAdd(Km + (bA + ia) * n + bD + id, x);
                    if (sPQ) atomicAdd(Km + (bD + id) * n + bA + ia, x);
                    continue;
                }
                r -= nK3;
                {  // with s12 and s34: K_jl += sum_ik G D_ik (and K_lj with sPQ)
                    if (!(s12 && s34)) continue;
                    const int ib = r / ND, id = r % ND;
                    double x = 0.0;
                    for (int ia = 0; ia < NA; ++ia)
                        for (int ic = 0; ic < NC; ++ic) x = fma(G(ia, ib, ic, id), Dv(bA + ia, bC + ic), x);
                    atomicAdd(Km + (bB + ib) * n + bD + id, x);
                    if (sPQ) atomicAdd(Km + (bD + id) * n + bB + ib, x);
                }
            }
        } else {
            for (int o = lane; o < W::NOUT; o += 32) {
                const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
                dense_images(a.out, n, P.bf1 + ia, P.bf2 + ib, Q.bf1 + ic, Q.bf2 + id, s12, s34, sPQ, H[__ldg(outs + o)]);
            }
        }
        return;
    }
    if (DERIV == 2 && mode == WMODE_HVP) {
        // Hessian-vector product of E = sum Gamma G with Gamma fixed: along v the
        // quartet moves by w_X = v(atom X) - v(atom D) for X = A, B, C (D by
        // invariance), so sum_V w_V h[U,V] is the directional derivative of the
        // first-derivative block U; contracted with Gamma it adds to the atom of U
        // and, with the opposite sign, to the atom of D.
        double wv[9], h9[9];
        const int atx[3] = {atA, atB, atC};
#pragma unroll
        for (int b = 0; b < 9; ++b) {
            wv[b] = __ldg(wa.dir + 3 * atx[b / 3] + b % 3) - __ldg(wa.dir + 3 * atD + b % 3);
            h9[b] = 0.0;
        }
        warp_hrr(W::hnodes(), W::hlev(), W::NHLEV, W::outs(), H, geo, lane, [&](int ob, double v) {
            int pidx = ob / W::NOUT;
            const int o = ob - pidx * W::NOUT;
            int Pc = 0;
            while (pidx >= 9 - Pc) {
                pidx -= 9 - Pc;
                ++Pc;
            }
            const int Qc = Pc + pidx;
            const double c = gam[o] * v;
            double wq = 0.0, wp = 0.0;
#pragma unroll
            for (int b = 0; b < 9; ++b) {
                wq = (b == Qc) ? wv[b] : wq;
                wp = (b == Pc) ? wv[b] : wp;
            }
#pragma unroll
            for (int b = 0; b < 9; ++b) {
                h9[b] += (b == Pc) ? c * wq : 0.0;
                h9[b] += (b == Qc && Pc != Qc) ? c * wp : 0.0;
            }
        });
#pragma unroll
        for (int b = 0; b < 9; ++b)
            for (int off = 16; off > 0; off >>= 1) h9[b] += __shfl_xor_sync(0xffffffffu, h9[b], off);
        if (lane == 0) {
            for (int x = 0; x < 3; ++x) {
                atomicAdd(wa.grad + 3 * atA + x, h9[x]);
                atomicAdd(wa.grad + 3 * atB + x, h9[3 + x]);
                atomicAdd(wa.grad + 3 * atC + x, h9[6 + x]);
                atomicAdd(wa.grad + 3 * atD + x, -(h9[x] + h9[3 + x] + h9[6 + x]));
            }
        }
        return;
    }
    if (DERIV == 2) {
        // 45 independent blocks h[U,V], U = 3X+i <= V = 3Y+j over the A, B, C
        // coordinates; with D = -(A+B+C) each h[U,V] adds to the nuclear Hessian
        // entries (U,V), (D_i,V), (U,D_j), (D_i,D_j) with signs +, -, -, +, for both
        // orderings of an off-diagonal block; an entry is kept in the unique
        // (nu1 <= nu2) slot of the reference's pair numbering.
        const int atoms[4] = {atA, atB, atC, atD};
        const long long n4 = n * n * n * n;
        const int M = wa.slice;  // dense: 3N; slice mode: packed pair (nu1 | nu2 << 16)
        warp_hrr(W::hnodes(), W::hlev(), W::NHLEV, W::outs(), H, geo, lane, [&](int ob, double v) {
            int pidx = ob / W::NOUT;
            const int o = ob - pidx * W::NOUT;
            int Pc = 0;
            while (pidx >= 9 - Pc) {
                pidx -= 9 - Pc;
                ++Pc;
            }
            const int Qc = Pc + pidx;
            const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
            const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
            for (int ord = 0; ord < (Pc == Qc ? 1 : 2); ++ord) {
                const int U = ord ? Qc : Pc, V = ord ? Pc : Qc;
                const int xu = U / 3, iu = U % 3, xv = V / 3, iv = V % 3;
                for (int su = 0; su < 2; ++su)
                    for (int sv = 0; sv < 2; ++sv) {
                        const int nu1 = 3 * atoms[su ? 3 : xu] + iu, nu2 = 3 * atoms[sv ? 3 : xv] + iv;
                        if (nu1 > nu2) continue;
                        const double c = ((su + sv) & 1) ? -v : v;
                        if (mode == WMODE_DER2_DENSE) {
                            const long long rank = (long long)nu1 * M - (long long)nu1 * (nu1 - 1) / 2 + (nu2 - nu1);
                            atomic_images_w(a.out + rank * n4, n, ii, jj, kk, ll, s12, s34, sPQ, c);
                        } else if (nu1 == (M & 0xffff) && nu2 == (M >> 16)) {
                            atomic_images_w(a.out, n, ii, jj, kk, ll, s12, s34, sPQ, c);
                        }
                    }
            }
        });
        return;
    }
    // derivative programs: the epilogue runs at each output node
    double g9[9];
#pragma unroll
    for (int b = 0; b < 9; ++b) g9[b] = 0.0;
    const int atoms[3] = {atA, atB, atC};
    const long long n4 = n * n * n * n;
    warp_hrr(W::hnodes(), W::hlev(), W::NHLEV, W::outs(), H, geo, lane, [&](int ob, double v) {
        const int blk = ob / W::NOUT, o = ob - blk * W::NOUT;
        if (mode == WMODE_GRAD) {
            const double c = gam[o] * v;
#pragma unroll
            for (int b = 0; b < 9; ++b) g9[b] += (b == blk) ? c : 0.0;
            return;
        }
        const int cen = blk / 3, xyz = blk - 3 * cen;
        const int atc = atoms[cen];
        if (atc == atD) return;
        const int id = o % ND, ic = (o / ND) % NC, ib = (o / (ND * NC)) % NB, ia = o / (ND * NC * NB);
        const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
        const int sp = 3 * atc + xyz, sm = 3 * atD + xyz;
        if (mode == WMODE_DER_TILE) {
            const long long e = qi * W::NOUT + o;
            tile_add(a.out, wa.tile_E, sp, e, wa.tile_images, s12, s34, sPQ, v);
            tile_add(a.out, wa.tile_E, sm, e, wa.tile_images, s12, s34, sPQ, -v);
            return;
        }
        if (mode == WMODE_DER_DENSE) {
            atomic_images_w(a.out + (long long)sp * n4, n, ii, jj, kk, ll, s12, s34, sPQ, v);
            atomic_images_w(a.out + (long long)sm * n4, n, ii, jj, kk, ll, s12, s34, sPQ, -v);
        } else {
            if (sp == wa.slice) atomic_images_w(a.out, n, ii, jj, kk, ll, s12, s34, sPQ, v);
            if (sm == wa.slice) atomic_images_w(a.out, n, ii, jj, kk, ll, s12, s34, sPQ, -v);
        }
    });
    if (mode == WMODE_GRAD) {
#pragma unroll
        for (int b = 0; b < 9; ++b)
            for (int off = 16; off > 0; off >>= 1) g9[b] += __shfl_xor_sync(0xffffffffu, g9[b], off);
        if (lane == 0) {
            for (int x = 0; x < 3; ++x) {
                atomicAdd(wa.grad + 3 * atA + x, g9[x]);
                atomicAdd(wa.grad + 3 * atB + x, g9[3 + x]);
                atomicAdd(wa.grad + 3 * atC + x, g9[6 + x]);
                atomicAdd(wa.grad + 3 * atD + x, -(g9[x] + g9[3 + x] + g9[6 + x]));
            }
        }
    }
}

template <class W, int DERIV>
void launch_warp(const WarpArgs& wa, int mode, cudaStream_t s) {
    const size_t smem = sizeof(double) * (size_t)W::SMEM_PER_WARP * WARP_QPB;
    auto k = k_warp<W, DERIV>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int qpb = WARP_QPB / wa.wpq;
    const long long nb = (wa.e.nq + qpb - 1) / qpb;
    if (nb) k<<<(unsigned)nb, WARP_QPB * 32, smem, s>>>(wa, mode);
}

typedef void (*WarpLaunch)(const WarpArgs&, int mode, cudaStream_t);

// VRR of one (quartet, primitive chunk) task per warp into the quartet's global
// accumulators; another kernel then runs the HRR from them.  For the classes with
// few quartets and long primitive loops (many warps per quartet keep the GPU
// full) and for the derivative classes whose accumulators and HRR slots do not
// fit a warp's shared memory.  Derivative programs (DER) map items to the
// cooperative engine's accumulator layout (nacc per quartet); plain programs keep
// the item order (NITEM_PAD per quartet).  Task quartet indices are relative to
// a.quartets; acc must be zeroed before the launch.
template <class W, bool DER, bool ITEMS = false>
__global__ void __launch_bounds__(WARP_QPB * 32) k_gvrr(EriArgs a, const int2* __restrict__ tasks, long long ntask,
                                                         int chunk, double* __restrict__ acc, int nacc) {
    const unsigned lane = threadIdx.x & 31;
    const long long ti = (long long)blockIdx.x * WARP_QPB + (threadIdx.x >> 5);
    if (ti >= ntask) return;  // whole warp
    const int2 task = tasks[ti];
    const int2 pq = a.quartets[task.x];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    if (DER && P.atom1 == P.atom2 && P.atom1 == Q.atom1 && P.atom1 == Q.atom2) return;  // reference skips these
    if (!DER && jk_screened(a, pq, P, Q)) return;  // J/K density screening (set only in J/K calls)
    // ITEMS: derivative items kept in item order (NITEM_PAD per quartet) for the
    // warp kernel's own HRR instead of the cooperative layout
    double* qacc = acc + (size_t)task.x * ((DER && !ITEMS) ? nacc : W::NITEM_PAD);
    const bool f32 = task.x >= a.nq64;  // warp-uniform: one task per warp
    // per-warp shared memory: [staged primitive pairs][mbarrier][chunk save area]
    extern __shared__ __align__(16) double wv_sm[];
    const int stage = a.prim_stage;
    const size_t per_warp = (size_t)stage * (sizeof(PrimPair) / 8) + 2 + W::SAVE;
    double* wbase = wv_sm + (size_t)(threadIdx.x >> 5) * per_warp;
    PrimPair* sp = reinterpret_cast<PrimPair*>(wbase);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(wbase + (size_t)stage * (sizeof(PrimPair) / 8));
    double* save = wbase + (size_t)stage * (sizeof(PrimPair) / 8) + 2;
    const PrimPair* bra = a.prims + P.prim_off;
    const PrimPair* ket = a.prims + Q.prim_off;
    if (stage) {
        // the quartet's bra and ket primitive pairs, one bulk copy each
        if (lane == 0) qx_mbar_init(bar, 1);
        __syncwarp();
        if (lane == 0) {
            const unsigned bb = (unsigned)(P.nprim * sizeof(PrimPair)), kb = (unsigned)(Q.nprim * sizeof(PrimPair));
            qx_mbar_expect_tx(bar, bb + kb);
            qx_bulk_g2s(sp, bra, bb, bar);
            qx_bulk_g2s(sp + P.nprim, ket, kb, bar);
        }
        if (!qx_mbar_wait(bar, 0, a.wait_limit)) {
            // report the timeout, then wait (bounded) for the copies to land so
            // none is still writing this block's shared memory when the warp exits
            if (lane == 0 && a.err) atomicOr(a.err, 1);
            qx_mbar_wait(bar, 0, 1 << 24);
            return;
        }
        bra = sp;
        ket = sp + P.nprim;
    }
    const int nk = Q.nprim, ntot = P.nprim * nk;
    const int tend = min(ntot, task.y + chunk);
    for (int t0 = task.y; t0 < tend; t0 += 32) {
        const int t = t0 + (int)lane;
        const bool act = t < tend;
        const int tt = act ? t : task.y;
        const int i = tt / nk, j = tt - i * nk;
        const PrimPair p = bra[i];
        const PrimPair r = ket[j];
        PrimQ q;
        double Fp[W::S + 1];
        prim_setup<W::S>(p, r, a.boys, q, Fp);
        if (!act) {
#pragma unroll
            for (int m = 0; m <= W::S; ++m) Fp[m] = 0.0;
        }
        const double wa = 2.0 * p.alpha, wb = 2.0 * (p.zeta - p.alpha), wc = 2.0 * r.alpha;
        if (f32) {
            float Ff[W::S + 1];
#pragma unroll
            for (int m = 0; m <= W::S; ++m) Ff[m] = (float)Fp[m];
            const PrimQT<float> qf = qx_to_float(q);
            float* sf = reinterpret_cast<float*>(save);
            if constexpr (DER && !ITEMS)
                W::vrr(Ff, qf, wa, wb, wc, GlobalSink{qacc, W::vmap()}, lane, sf);
            else
                W::vrr(Ff, qf, wa, wb, wc, IdentSink{qacc}, lane, sf);
        } else {
            if constexpr (DER && !ITEMS)
                W::vrr(Fp, q, wa, wb, wc, GlobalSink{qacc, W::vmap()}, lane, save);
            else
                W::vrr(Fp, q, wa, wb, wc, IdentSink{qacc}, lane, save);
        }
        __syncwarp();
    }
}

template <class W, bool DER, bool ITEMS = false>
void launch_gvrr(const EriArgs& a, const int2* tasks, long long ntask, int chunk, double* acc, int nacc,
                 cudaStream_t s) {
    const long long nb = (ntask + WARP_QPB - 1) / WARP_QPB;
    const size_t per_warp = (size_t)a.prim_stage * (sizeof(PrimPair) / 8) + 2 + W::SAVE;
    const size_t smem = sizeof(double) * per_warp * WARP_QPB;
    auto k = k_gvrr<W, DER, ITEMS>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (nb) k<<<(unsigned)nb, WARP_QPB * 32, smem, s>>>(a, tasks, ntask, chunk, acc, nacc);
}

typedef void (*WvrrLaunch)(const EriArgs&, const int2*, long long, int, double*, int, cudaStream_t);

}  // namespace qx
