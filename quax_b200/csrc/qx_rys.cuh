// qx_rys.cuh -- Rys-quadrature engine: every class up to (ff|ff), and nuclear
// derivatives of any order, through one looped design.
//
// Method (published mathematics, written here):
//   * A primitive integral is pref * sum_r w_r Ix(u_r) Iy(u_r) Iz(u_r), with
//     (u_r, w_r) the n-point Gauss rule of the measure e^{-T u} u^{-1/2}/2 du on
//     [0, 1] (moments F_m(T)), n = floor(L/2) + 1 for total angular momentum L
//     (M. Dupuis, J. Rys & H. F. King, J. Chem. Phys. 65, 111 (1976); J. Rys,
//     M. Dupuis & H. F. King, J. Comput. Chem. 4, 154 (1983)).  Nodes and
//     weights come from the tabulated Chebyshev series of qx_rys_table.inc.
//   * The 1-D factors I(i, k) (i quanta on the bra, k on the ket, one Cartesian
//     direction, one root) follow the two-term recurrences
//       I(i+1, k) = C00 I(i, k) + i B10 I(i-1, k) + k B00 I(i, k-1)
//       I(i, k+1) = D00 I(i, k) + k B01 I(i, k-1) + i B00 I(i-1, k)
//     with B00 = u/(2(p+q)), B10 = (1 - u q/(p+q))/(2p), B01 = (1 - u p/(p+q))/(2q),
//     C00 = (P-A) - u q (P-Q)/(p+q), D00 = (Q-C) + u p (P-Q)/(p+q)
//     (the Obara-Saika coefficients with the (m+1) index replaced by a factor u),
//     then the transfer I(a, b+1) = I(a+1, b) + (A-B) I(a, b) on each side
//     (Head-Gordon & Pople, J. Chem. Phys. 89, 5777 (1988), in one dimension).
//   * Derivatives act on one direction's factor: d/dA_x g_a = 2 alpha g_{a+1} -
//     a g_{a-1} (applied k times for order k), so every derivative integral is a
//     product of three 1-D tables.
//
// Device organisation: a team of TS threads (one warp, or 2..8 warps with named
// barriers) owns one contracted quartet at a time and walks its primitive
// quartets.  Per primitive quartet: 2n threads evaluate the nodes/weights, then
// per batch of RB roots the 3*RB (direction, root) units build their 2-D tables
// (one thread per unit) and the transfer levels run -- in parallel over the team
// level by level, or, for small units, the whole unit in the thread that built
// its 2-D table -- the derivative tables are formed (higher-order kinds; the
// first-derivative kinds form dA, dB, dC from the raw table inside the
// products), and every thread adds the products for its own Cartesian
// components into registers.  All tables live in shared memory; nothing is
// written to global memory until the epilogue.
#pragma once
#include "qx_warp.cuh"
#include "qx_rys_table.inc"

#ifdef __CUDACC__
#define QX_HD __host__ __device__
#else
#define QX_HD
#endif

namespace qx {

constexpr int kRysTmax[QX_RYS_NMAX + 1] = {QX_RYS_TMAX_LIST};
constexpr int kRysOff[QX_RYS_NMAX + 1] = {QX_RYS_OFF_LIST};
constexpr int RYS_TABLE_DOUBLES = QX_RYS_TAB_SIZE + 2 * QX_RYS_ASYM_SIZE;

// Kinds of Rys programs: which centres are raised for derivatives, the
// derivative order the quadrature must integrate, and the per-direction 1-D
// derivative tables the products read.
enum { RK_PLAIN = 0, RK_GRAD = 1, RK_HVP = 2, RK_GRADT = 3, RK_GRADL = 4, RK_DER1 = 11, RK_DER2 = 12,
       RK_DER3 = 13, RK_DER4 = 14 };
// The adjoint-gradient kinds: RK_GRADL is RK_GRAD with every unit's tables built
// level by level over the team (the autotuner picks the faster build per class).
QX_HD constexpr bool rys_is_grad(int kind) { return kind == RK_GRAD || kind == RK_GRADL; }
// Epilogues of the plain kind (the derivative kinds have their own).
enum { RMODE_DENSE = 0, RMODE_UNIQUE = 1, RMODE_SCHWARZ = 2, RMODE_JK = 3 };

QX_HD constexpr int rys_binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

template <int KIND>
struct RysKind {  // RK_DERk: all four centres raised by k, every op with total order <= k
    static constexpr int ORD = KIND - 10;
    static constexpr int KA = ORD, KB = ORD, KC = ORD, KD = ORD;
    static constexpr int NOPS = rys_binom(ORD + 4, 4);
};
template <>
struct RysKind<RK_PLAIN> {
    static constexpr int ORD = 0, KA = 0, KB = 0, KC = 0, KD = 0, NOPS = 0;
};
template <>
struct RysKind<RK_GRAD> {  // A, B, C raised by one; dA, dB, dC formed in the products (D by invariance)
    static constexpr int ORD = 1, KA = 1, KB = 1, KC = 1, KD = 0, NOPS = 0;
};
template <>
struct RysKind<RK_GRADL> : RysKind<RK_GRAD> {};
template <>
struct RysKind<RK_GRADT> {  // as RK_GRAD, but the 9 derivative integrals are written to a tile
    static constexpr int ORD = 1, KA = 1, KB = 1, KC = 1, KD = 0, NOPS = 0;
};
template <>
struct RysKind<RK_HVP> {  // A, B, C raised by two; tables I, dA, dB, dC, V, dA V, dB V, dC V
    static constexpr int ORD = 2, KA = 2, KB = 2, KC = 2, KD = 0, NOPS = 8;
};

// Shared memory per block the engine may plan for (leaves room for two blocks
// per SM when a class fits; the largest kinds take one block per SM).
constexpr int RYS_SMEM_TARGET = 100 * 1024;
constexpr int RYS_SMEM_MAX = 227 * 1024;
constexpr int RYS_HDR = 128;       // per team: nodes/weights (32), reductions (80), spare
constexpr int RYS_CHMAX = 64;      // derivative multi-indices per work item (RK_DERk)
constexpr int RYS_DERK_HDR = 3 * RYS_CHMAX;

template <int LA, int LB, int LC, int LD, int KIND>
struct RysCls {
    using K = RysKind<KIND>;
    static constexpr int NA = ncart_h(LA), NB = ncart_h(LB), NC = ncart_h(LC), ND = ncart_h(LD);
    static constexpr int NCOMP = NA * NB * NC * ND;
    static constexpr int A1 = LA + K::KA + 1, B1 = LB + K::KB + 1, C1 = LC + K::KC + 1, D1 = LD + K::KD + 1;
    static constexpr int NI = A1 + B1 - 1, NK = C1 + D1 - 1;
    static constexpr int NR = (LA + LB + LC + LD + K::ORD) / 2 + 1;
    static_assert(NR <= QX_RYS_NMAX, "Rys table too short for this class");
    static constexpr int SBRA = B1 * NI * NK;       // bra transfer levels [b][a][k]
    static constexpr int SRAW = A1 * B1 * D1 * NK;  // ket transfer levels [a][b][d][c]
    static constexpr int USZ = SBRA + SRAW;          // one (direction, root) unit
    static constexpr int SZ0 = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    static constexpr int NOPS = K::NOPS;
    static constexpr int UOPS = NOPS * SZ0;
    // team size: about 12 components per thread (8 for the gradient tile, which
    // keeps 9 sums per component), 32..256 threads
    static constexpr int TS0 = KIND == RK_GRADT ? (NCOMP + 7) / 8 : (NCOMP + 11) / 12;
    static constexpr int TS1 = TS0 <= 32 ? 32 : TS0 <= 64 ? 64 : TS0 <= 128 ? 128 : 256;
    static constexpr int HDR = RYS_HDR + (KIND >= RK_DER1 ? RYS_DERK_HDR : 0);
    static constexpr int PER_ROOT = 3 * (USZ + UOPS);
    // one root per batch with (128 / TS1) teams per block must fit; otherwise the
    // block holds a single team of 128 threads (the large derivative kinds)
    static constexpr bool MULTI = TS1 >= 128 || (128 / TS1) * (HDR + PER_ROOT) * 8 <= RYS_SMEM_MAX;
    static constexpr int TS = MULTI ? TS1 : 128;
    static constexpr int BS = TS < 128 ? 128 : TS;
    static constexpr int TPB = BS / TS;
    static constexpr int NCPT = (NCOMP + TS - 1) / TS;
    static constexpr int RB0 = (RYS_SMEM_TARGET / 8 / TPB - HDR) / PER_ROOT;
    static constexpr int RB = RB0 < 1 ? 1 : (RB0 > NR ? NR : RB0);
    static constexpr int TEAM_SMEM = HDR + RB * PER_ROOT;  // doubles
    static constexpr int SMEM = TPB * TEAM_SMEM * 8;       // bytes per block
    static constexpr bool FITS = SMEM <= RYS_SMEM_MAX;
    // minimum blocks per SM for the register budget: one for the 256-thread
    // classes, which need the full 255 registers (left to its own heuristics the
    // compiler gives some of them 64-80 registers and kilobytes of spills, and
    // those builds returned wrong gradients for (33|32)); the compiler's choice
    // (0) for 128-thread blocks, measured faster than capping them at 170
    // registers for three blocks per SM
    static constexpr int MINB = BS >= 256 ? 1 : 0;
    // offsets of one component in a table are packed 10 bits per direction
    // products read the raw transferred table (plain and gradient kinds) or the
    // op tables (the others)
    static constexpr bool RAW = KIND == RK_PLAIN || rys_is_grad(KIND) || KIND == RK_GRADT;
    static_assert((!RAW || SRAW < 1024) && SZ0 < 1024, "1-D table offsets exceed 10 bits");
    // one thread builds a whole (direction, root) unit -- 2-D table and both
    // transfers -- when the units keep at least a sixth of the team busy or are small
    static constexpr bool SEQ = KIND != RK_GRADL && (6 * RB >= TS || SRAW <= 160);
    // derivative tensors: multi-indices accumulated per pass over the primitives
    static constexpr int MG = NCPT >= 32 ? 1 : (32 / NCPT > 8 ? 8 : 32 / NCPT);
    // gradient tile: derivative coordinates (of the 9) accumulated per pass
    static constexpr int GG = NCPT * 9 <= 72 ? 9 : (72 / NCPT < 1 ? 1 : 72 / NCPT);
};

struct RysArgs {
    EriArgs e;
    const double* rys = nullptr;  // device table: QX_RYS_TAB | asymptotic y | asymptotic W
    // adjoint gradient and Hessian-vector product
    const double* D = nullptr;
    double cj = 0.0, ck = 0.0;
    double* grad = nullptr;       // 3N output (atomic adds)
    const double* dir = nullptr;  // HVP direction (3N)
    // derivative tensors (RK_DERk): dense (slice_k == 0) or one slice
    int M = 0;                    // 3N
    int chunk = 1;                // multi-indices per work item
    int nchunk = 1;               // work items per quartet
    int slice_k = 0;              // 0: dense; else the slice's order (== k)
    int slice_nu[4] = {0, 0, 0, 0};  // the slice's sorted nuclear indices
    // first-derivative tile (RK_DER1 only): out is a (3N, tile_E) row-major
    // buffer with the layout of the warp kernels' WMODE_DER_TILE
    long long tile_E = 0;
    int tile_images = 0;
};

// ------------------------------------------------------------ nodes, weights ---
// Function f of the n-point rule at T: nodes f = 0..n-1, weights f = n..2n-1.
template <int N>
QX_HD inline double rys_fn(const double* __restrict__ rt, int f, double T) {
    constexpr double TM = kRysTmax[N];
    constexpr int OFF = kRysOff[N];
    if (T < TM) {
        const int i = (int)(0.5 * T);
        const double x = T - (2.0 * i + 1.0);
        const double* __restrict__ c = rt + OFF + (i * 2 * N + f) * QX_RYS_NCOEF;
        const double x2 = 2.0 * x;
        double b1 = 0.0, b2 = 0.0;
#pragma unroll
        for (int k = QX_RYS_NCOEF - 1; k >= 1; --k) {
            const double t = fma(x2, b1, c[k] - b2);
            b2 = b1;
            b1 = t;
        }
        return fma(x, b1, c[0] - b2);
    }
    const double* __restrict__ ay = rt + QX_RYS_TAB_SIZE;
    constexpr int o = N * (N - 1) / 2;
    if (f < N) return ay[o + f] / T;
    return ay[QX_RYS_ASYM_SIZE + o + f - N] * 0.5 / sqrt(T);
}

// Per-primitive-quartet scalars.
struct RysPrim {
    double PA[3], QC[3], PQ[3], AB[3], CD[3];
    double p, q, rs;  // rs = 1/(p+q)
    double T, pref;
    double e2[4];  // 2 alpha, 2 beta, 2 gamma, 2 delta
};

QX_HD inline void rys_prim(const PrimPair& a, const PrimPair& c, const PairInfo& P, const PairInfo& Q, RysPrim& s) {
    s.p = a.zeta;
    s.q = c.zeta;
    const double ze = a.zeta + c.zeta;
    s.rs = 1.0 / ze;
    s.PA[0] = a.PAx; s.PA[1] = a.PAy; s.PA[2] = a.PAz;
    s.QC[0] = c.PAx; s.QC[1] = c.PAy; s.QC[2] = c.PAz;
    s.PQ[0] = a.Px - c.Px; s.PQ[1] = a.Py - c.Py; s.PQ[2] = a.Pz - c.Pz;
    s.AB[0] = P.ABx; s.AB[1] = P.ABy; s.AB[2] = P.ABz;
    s.CD[0] = Q.ABx; s.CD[1] = Q.ABy; s.CD[2] = Q.ABz;
    const double rho = a.zeta * c.zeta * s.rs;
    s.T = rho * (s.PQ[0] * s.PQ[0] + s.PQ[1] * s.PQ[1] + s.PQ[2] * s.PQ[2]);
    s.pref = a.K * c.K * sqrt(s.rs);
    s.e2[0] = 2.0 * a.alpha;
    s.e2[1] = 2.0 * (a.zeta - a.alpha);
    s.e2[2] = 2.0 * c.alpha;
    s.e2[3] = 2.0 * (c.zeta - c.alpha);
}

// Cartesian exponents of component i of a shell of angular momentum l
// (Libint standard order: x^l, x^{l-1}y, x^{l-1}z, ...).
QX_HD inline void cart_exps(int l, int i, int& lx, int& ly, int& lz) {
    lx = l;
    int rem = i;
    while (rem > l - lx) {
        rem -= l - lx + 1;
        --lx;
    }
    ly = l - lx - rem;
    lz = rem;
}

// 1-D derivative operator (d/dX)^k on the Gaussian index i with e2 = 2 * exponent:
// d g_i = e2 g_{i+1} - i g_{i-1}.  cf[j] multiplies g_{i + 2j - k}, j = 0..k.
QX_HD inline void rys_dexp(int k, int i, double e2, double* cf) {
    double c[5] = {1.0, 0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < k; ++s) {
        double nc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int j = 0; j <= s; ++j) {
            const int sh = 2 * j - s;
            nc[j + 1] += e2 * c[j];
            nc[j] -= (double)(i + sh) * c[j];
        }
        for (int j = 0; j < 5; ++j) c[j] = nc[j];
    }
    for (int j = 0; j <= k; ++j) cf[j] = c[j];
}

// Rank of (ka, kb, kc, kd), all >= 0 with sum <= K, among such tuples in
// lexicographic order (the op-table index of the RK_DERk kinds).
QX_HD inline int rys_op_rank(int K, int ka, int kb, int kc, int kd) {
    int r = 0;
    for (int v = 0; v < ka; ++v) r += rys_binom(K - v + 3, 3);
    for (int v = 0; v < kb; ++v) r += rys_binom(K - ka - v + 2, 2);
    for (int v = 0; v < kc; ++v) r += rys_binom(K - ka - kb - v + 1, 1);
    return r + kd;
}

// Rank of a non-decreasing k-tuple of values in [0, n) among all such tuples in
// lexicographic order -- the reference's numbering of unique derivatives
// (combinations with repetition, quax/integrals/utils.h:158-172).
QX_HD inline long long rys_multiset_rank(const int* v, int k, int n) {
    long long r = 0;
    int prev = 0;
    for (int i = 0; i < k; ++i) {
        for (int x = prev; x < v[i]; ++x) r += rys_binom(n - x + k - i - 2, k - i - 1);
        prev = v[i];
    }
    return r;
}

// The m-th non-decreasing k-tuple over [0, n) (inverse of rys_multiset_rank).
QX_HD inline void rys_multiset_unrank(long long m, int k, int n, int* v) {
    int prev = 0;
    for (int i = 0; i < k; ++i) {
        for (int x = prev; x < n; ++x) {
            const long long c = rys_binom(n - x + k - i - 2, k - i - 1);
            if (m < c) {
                v[i] = x;
                prev = x;
                break;
            }
            m -= c;
        }
    }
}

// ------------------------------------------------------------------ phases ---
// Each phase processes elements tid, tid + nth, ... of its index space; the
// device runs them over a team with a barrier after each, the host check runs
// them with (0, 1).
//
// Unit u = 3 * (root within batch) + direction; U holds nrb * 3 units of USZ.
template <class C>
QX_HD inline double& rys_gb(double* U, int u, int b, int a, int k) {
    return U[(size_t)u * C::USZ + (b * C::NI + a) * C::NK + k];
}
template <class C>
QX_HD inline double& rys_gk(double* U, int u, int a, int b, int d, int c) {
    return U[(size_t)u * C::USZ + C::SBRA + ((a * C::B1 + b) * C::D1 + d) * C::NK + c];
}

// 2-D tables, one thread per unit.  The weight (times pref) goes into z.
template <class C>
QX_HD inline void rys_phase_2d(const RysPrim& s, const double* uw, int rb0, int nrb, double* U, int tid, int nth) {
    for (int u = tid; u < 3 * nrb; u += nth) {
        const int x = u % 3, r = rb0 + u / 3;
        const double t2 = uw[r];
        const double B00 = 0.5 * t2 * s.rs;
        const double B10 = 0.5 / s.p * (1.0 - t2 * s.q * s.rs);
        const double B01 = 0.5 / s.q * (1.0 - t2 * s.p * s.rs);
        const double C00 = s.PA[x] - t2 * s.q * s.rs * s.PQ[x];
        const double D00 = s.QC[x] + t2 * s.p * s.rs * s.PQ[x];
        double* g = U + (size_t)u * C::USZ;  // level b = 0: g[i * NK + k]
        g[0] = x == 2 ? uw[C::NR + r] : 1.0;
        if (C::NI > 1) g[C::NK] = C00 * g[0];
        for (int i = 2; i < C::NI; ++i) g[i * C::NK] = C00 * g[(i - 1) * C::NK] + (i - 1) * B10 * g[(i - 2) * C::NK];
        for (int k = 1; k < C::NK; ++k) {
            const double kB01 = (k - 1) * B01;
            g[k] = D00 * g[k - 1] + (k > 1 ? kB01 * g[k - 2] : 0.0);
            for (int i = 1; i < C::NI; ++i)
                g[i * C::NK + k] = D00 * g[i * C::NK + k - 1] + (k > 1 ? kB01 * g[i * C::NK + k - 2] : 0.0) +
                                   i * B00 * g[(i - 1) * C::NK + k - 1];
        }
    }
}

// Bra transfer level b: I(a, b) = I(a+1, b-1) + AB I(a, b-1), a < NI - b.
template <class C>
QX_HD inline void rys_phase_bra(const RysPrim& s, int b, int nrb, double* U, int tid, int nth) {
    const int na = C::NI - b, per = na * C::NK;
    for (int e = tid; e < 3 * nrb * per; e += nth) {
        const int u = e / per, rest = e - u * per, a = rest / C::NK, k = rest - a * C::NK;
        rys_gb<C>(U, u, b, a, k) = rys_gb<C>(U, u, b - 1, a + 1, k) + s.AB[u % 3] * rys_gb<C>(U, u, b - 1, a, k);
    }
}

// Ket level 0 (copy of the bra-transferred table) and level d:
// I(c, d) = I(c+1, d-1) + CD I(c, d-1), c < NK - d.
template <class C>
QX_HD inline void rys_phase_ket(const RysPrim& s, int d, int nrb, double* U, int tid, int nth) {
    const int nc = C::NK - d, per = C::A1 * C::B1 * nc;
    for (int e = tid; e < 3 * nrb * per; e += nth) {
        const int u = e / per;
        int rest = e - u * per;
        const int a = rest / (C::B1 * nc);
        rest -= a * C::B1 * nc;
        const int b = rest / nc, c = rest - b * nc;
        if (d == 0)
            rys_gk<C>(U, u, a, b, 0, c) = rys_gb<C>(U, u, b, a, c);
        else
            rys_gk<C>(U, u, a, b, d, c) =
                rys_gk<C>(U, u, a, b, d - 1, c + 1) + s.CD[u % 3] * rys_gk<C>(U, u, a, b, d - 1, c);
    }
}

// The whole unit in one thread: 2-D table, bra and ket transfers, with plain
// incrementing loops (the level-parallel phases above decode every element's
// indices, which costs more than the arithmetic for small units).
template <class C>
QX_HD inline void rys_phase_units(const RysPrim& s, const double* uw, int rb0, int nrb, double* U, int tid, int nth) {
    for (int u = tid; u < 3 * nrb; u += nth) {
        const int x = u % 3, r = rb0 + u / 3;
        const double t2 = uw[r];
        const double B00 = 0.5 * t2 * s.rs;
        const double B10 = 0.5 / s.p * (1.0 - t2 * s.q * s.rs);
        const double B01 = 0.5 / s.q * (1.0 - t2 * s.p * s.rs);
        const double C00 = s.PA[x] - t2 * s.q * s.rs * s.PQ[x];
        const double D00 = s.QC[x] + t2 * s.p * s.rs * s.PQ[x];
        const double AB = s.AB[x], CD = s.CD[x];
        double* g = U + (size_t)u * C::USZ;  // level b: g[(b * NI + a) * NK + k]
        g[0] = x == 2 ? uw[C::NR + r] : 1.0;
        if (C::NI > 1) g[C::NK] = C00 * g[0];
        for (int i = 2; i < C::NI; ++i) g[i * C::NK] = C00 * g[(i - 1) * C::NK] + (i - 1) * B10 * g[(i - 2) * C::NK];
        for (int k = 1; k < C::NK; ++k) {
            const double kB01 = (k - 1) * B01;
            g[k] = D00 * g[k - 1] + (k > 1 ? kB01 * g[k - 2] : 0.0);
            for (int i = 1; i < C::NI; ++i)
                g[i * C::NK + k] = D00 * g[i * C::NK + k - 1] + (k > 1 ? kB01 * g[i * C::NK + k - 2] : 0.0) +
                                   i * B00 * g[(i - 1) * C::NK + k - 1];
        }
        for (int b = 1; b < C::B1; ++b) {
            const double* gp = g + (b - 1) * C::NI * C::NK;
            double* gc = g + b * C::NI * C::NK;
            for (int a = 0; a < C::NI - b; ++a)
                for (int k = 0; k < C::NK; ++k) gc[a * C::NK + k] = gp[(a + 1) * C::NK + k] + AB * gp[a * C::NK + k];
        }
        double* h = g + C::SBRA;  // [a][b][d][c]
        for (int a = 0; a < C::A1; ++a)
            for (int b = 0; b < C::B1; ++b) {
                double* hb = h + (a * C::B1 + b) * C::D1 * C::NK;
                const double* src = g + (b * C::NI + a) * C::NK;
                for (int c = 0; c < C::NK; ++c) hb[c] = src[c];
                for (int d = 1; d < C::D1; ++d)
                    for (int c = 0; c < C::NK - d; ++c)
                        hb[d * C::NK + c] = hb[(d - 1) * C::NK + c + 1] + CD * hb[(d - 1) * C::NK + c];
            }
    }
}

// One op (per-centre derivative orders k[4]) of a unit at the unraised point
// (a, b, c, d) from the raised table.
template <class C>
QX_HD inline double rys_op_value(const RysPrim& s, double* U, int u, const int* k, int a, int b, int c, int d) {
    double ca[5], cb[5], cc[5], cd[5];
    rys_dexp(k[0], a, s.e2[0], ca);
    rys_dexp(k[1], b, s.e2[1], cb);
    rys_dexp(k[2], c, s.e2[2], cc);
    rys_dexp(k[3], d, s.e2[3], cd);
    double v = 0.0;
    for (int ja = 0; ja <= k[0]; ++ja) {
        const int ia = a + 2 * ja - k[0];
        if (ia < 0 || ca[ja] == 0.0) continue;
        for (int jb = 0; jb <= k[1]; ++jb) {
            const int ib = b + 2 * jb - k[1];
            if (ib < 0 || cb[jb] == 0.0) continue;
            for (int jc = 0; jc <= k[2]; ++jc) {
                const int ic = c + 2 * jc - k[2];
                if (ic < 0 || cc[jc] == 0.0) continue;
                const double cabc = ca[ja] * cb[jb] * cc[jc];
                for (int jd = 0; jd <= k[3]; ++jd) {
                    const int id = d + 2 * jd - k[3];
                    if (id < 0 || cd[jd] == 0.0) continue;
                    v += cabc * cd[jd] * rys_gk<C>(U, u, ia, ib, id, ic);
                }
            }
        }
    }
    return v;
}

// Op tables of the derivative kinds: O holds per unit NOPS tables of SZ0
// entries [a][b][c][d] (unraised extents).  RK_DERk: every (ka, kb, kc, kd)
// with sum <= k in rys_op_rank order; RK_HVP: I, dA, dB, dC, V, dA V, dB V, dC V
// with V = sum_X w_X dX along the direction w (per unit direction:
// w9[3 * X + direction]).
template <class C, int KIND, int LA, int LB, int LC, int LD>
QX_HD inline void rys_phase_ops(const RysPrim& s, int nrb, double* U, double* O, const double* w9, int tid, int nth) {
    constexpr int per = C::NOPS * C::SZ0;
    for (int e = tid; e < 3 * nrb * per; e += nth) {
        const int u = e / per;
        const int rest = e - u * per, op = rest / C::SZ0, el = rest - op * C::SZ0;
        const int d = el % (LD + 1), c = (el / (LD + 1)) % (LC + 1), b = (el / ((LD + 1) * (LC + 1))) % (LB + 1),
                  a = el / ((LD + 1) * (LC + 1) * (LB + 1));
        double v;
        if constexpr (KIND == RK_HVP) {
            // first and second derivatives on A, B, C in closed form: per centre the
            // index shifts by +-1 (+-2 for a repeated centre) with the factors of
            // d g_i = e2 g_{i+1} - i g_{i-1}
            const int x = u % 3;
            const int idx0[3] = {a, b, c};
            auto R = [&](const int* ix) { return rys_gk<C>(U, u, ix[0], ix[1], d, ix[2]); };
            auto d1 = [&](int X) {  // dX I
                int ix[3] = {a, b, c};
                ix[X] += 1;
                double r = s.e2[X] * R(ix);
                if (idx0[X]) {
                    ix[X] -= 2;
                    r -= idx0[X] * R(ix);
                }
                return r;
            };
            auto d2 = [&](int X, int Y) {  // dX dY I
                int ix[3] = {a, b, c};
                if (X == Y) {
                    const int i = idx0[X];
                    ix[X] = i + 2;
                    double r = s.e2[X] * s.e2[X] * R(ix);
                    ix[X] = i;
                    r -= s.e2[X] * (2 * i + 1) * R(ix);
                    if (i >= 2) {
                        ix[X] = i - 2;
                        r += (double)(i * (i - 1)) * R(ix);
                    }
                    return r;
                }
                double r = 0.0;
                for (int sx = 0; sx < 2; ++sx)
                    for (int sy = 0; sy < 2; ++sy) {
                        const int ixx = idx0[X] + (sx ? -1 : 1), iyy = idx0[Y] + (sy ? -1 : 1);
                        if (ixx < 0 || iyy < 0) continue;
                        const double cf = (sx ? -(double)idx0[X] : s.e2[X]) * (sy ? -(double)idx0[Y] : s.e2[Y]);
                        int jx[3] = {a, b, c};
                        jx[X] = ixx;
                        jx[Y] = iyy;
                        r += cf * R(jx);
                    }
                return r;
            };
            if (op == 0) {
                v = R(idx0);
            } else if (op < 4) {
                v = d1(op - 1);
            } else if (op == 4) {
                v = w9[x] * d1(0) + w9[3 + x] * d1(1) + w9[6 + x] * d1(2);
            } else {
                const int Y = op - 5;
                v = w9[x] * d2(0, Y) + w9[3 + x] * d2(1, Y) + w9[6 + x] * d2(2, Y);
            }
        } else if constexpr (C::K::ORD == 1) {
            // order 1, all four centres raised: ops in rys_op_rank order are
            // I, dD, dC, dB, dA, in closed form
            auto R = [&](int ia, int ib, int ic, int id) { return rys_gk<C>(U, u, ia, ib, id, ic); };
            if (op == 0) v = R(a, b, c, d);
            else if (op == 1) v = s.e2[3] * R(a, b, c, d + 1) - (d ? d * R(a, b, c, d - 1) : 0.0);
            else if (op == 2) v = s.e2[2] * R(a, b, c + 1, d) - (c ? c * R(a, b, c - 1, d) : 0.0);
            else if (op == 3) v = s.e2[1] * R(a, b + 1, c, d) - (b ? b * R(a, b - 1, c, d) : 0.0);
            else v = s.e2[0] * R(a + 1, b, c, d) - (a ? a * R(a - 1, b, c, d) : 0.0);
        } else {
            constexpr int K = C::K::ORD;
            // unrank op within tuples of sum <= K (lexicographic)
            int k[4];
            int r = op;
            int left = K;
            for (int pos = 0; pos < 3; ++pos) {
                int val = 0;
                for (;;) {
                    const int cnt = rys_binom(left - val + 3 - pos, 3 - pos);
                    if (r < cnt) break;
                    r -= cnt;
                    ++val;
                }
                k[pos] = val;
                left -= val;
            }
            k[3] = r;
            v = rys_op_value<C>(s, U, u, k, a, b, c, d);
        }
        O[(size_t)u * per + op * C::SZ0 + el] = v;
    }
}

// Packed offsets of component kc in the three directions' tables: the raw
// transferred table for the plain kind, the op tables (unraised [a][b][c][d])
// for the derivative kinds.
template <class C, int LA, int LB, int LC, int LD, bool RAW>
QX_HD inline int rys_comp_offsets(int kc) {
    constexpr int NB = C::NB, NC = C::NC, ND = C::ND;
    const int id = kc % ND, ic = (kc / ND) % NC, ib = (kc / (ND * NC)) % NB, ia = kc / (ND * NC * NB);
    int ea[3], eb[3], ec[3], ed[3];
    cart_exps(LA, ia, ea[0], ea[1], ea[2]);
    cart_exps(LB, ib, eb[0], eb[1], eb[2]);
    cart_exps(LC, ic, ec[0], ec[1], ec[2]);
    cart_exps(LD, id, ed[0], ed[1], ed[2]);
    int packed = 0;
    for (int x = 0; x < 3; ++x) {
        const int o = RAW ? ((ea[x] * C::B1 + eb[x]) * C::D1 + ed[x]) * C::NK + ec[x]
                          : ((ea[x] * (LB + 1) + eb[x]) * (LC + 1) + ec[x]) * (LD + 1) + ed[x];
        packed |= o << (10 * x);
    }
    return packed;
}

// Cartesian exponents (a, b, c) of component kc in the three directions, packed
// 2 bits each, 6 bits per direction (the factors of d g_i = 2e g_{i+1} - i g_{i-1}).
template <class C, int LA, int LB, int LC, int LD>
QX_HD inline int rys_comp_exps(int kc) {
    constexpr int NB = C::NB, NC = C::NC, ND = C::ND;
    const int ic = (kc / ND) % NC, ib = (kc / (ND * NC)) % NB, ia = kc / (ND * NC * NB);
    int ea[3], eb[3], ec[3];
    cart_exps(LA, ia, ea[0], ea[1], ea[2]);
    cart_exps(LB, ib, eb[0], eb[1], eb[2]);
    cart_exps(LC, ic, ec[0], ec[1], ec[2]);
    int p = 0;
    for (int x = 0; x < 3; ++x) p |= (ea[x] | eb[x] << 2 | ec[x] << 4) << (6 * x);
    return p;
}

// First derivatives of one direction's factor from the raw table at offset o
// (exponents e = a | b << 2 | c << 4): dA, dB, dC.
template <class C>
QX_HD inline void rys_raw_d1(const double* T, int o, int e, const double* e2, double& dA, double& dB, double& dC) {
    constexpr int SA = C::B1 * C::D1 * C::NK, SB = C::D1 * C::NK;
    const int a = e & 3, b = (e >> 2) & 3, c = (e >> 4) & 3;
    dA = e2[0] * T[o + SA];
    if (a) dA -= a * T[o - SA];
    dB = e2[1] * T[o + SB];
    if (b) dB -= b * T[o - SB];
    dC = e2[2] * T[o + 1];
    if (c) dC -= c * T[o - 1];
}

// Plain kind: add the batch's products of component kc (packed offsets).
template <class C>
QX_HD inline double rys_prod_plain(const double* U, int nrb, int off) {
    const int ox = off & 1023, oy = (off >> 10) & 1023, oz = off >> 20;
    double s = 0.0;
    for (int r = 0; r < nrb; ++r) {
        const double* b = U + (size_t)3 * r * C::USZ + C::SBRA;
        s = fma(b[ox] * b[C::USZ + oy], b[2 * C::USZ + oz], s);
    }
    return s;
}

// Gradient kind: g[3X + i] += gam * sum_r (dX I)_i prod_{j != i} I_j, X = A, B, C,
// the derivatives formed from the raw tables of the batch's units.
template <class C>
QX_HD inline void rys_prod_grad(const double* U, int nrb, int off, int ex, const double* e2, double gam, double* g) {
    const int o[3] = {off & 1023, (off >> 10) & 1023, off >> 20};
    for (int r = 0; r < nrb; ++r) {
        const double* T = U + (size_t)3 * r * C::USZ + C::SBRA;
        const double I[3] = {T[o[0]], T[C::USZ + o[1]], T[2 * C::USZ + o[2]]};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            double dA, dB, dC;
            rys_raw_d1<C>(T + x * C::USZ, o[x], (ex >> (6 * x)) & 63, e2, dA, dB, dC);
            const double w = gam * (x == 0 ? I[1] * I[2] : (x == 1 ? I[0] * I[2] : I[0] * I[1]));
            g[x] = fma(dA, w, g[x]);
            g[3 + x] = fma(dB, w, g[3 + x]);
            g[6 + x] = fma(dC, w, g[6 + x]);
        }
    }
}

// Gradient-tile kind: acc[b - b0] += sum_r (dX I)_i prod_{j != i} I_j for the
// derivative coordinates b = 3X + i in [b0, b0 + GG).
template <class C>
QX_HD inline void rys_prod_gradt(const double* U, int nrb, int off, int ex, const double* e2, int b0, double* acc) {
    const int o[3] = {off & 1023, (off >> 10) & 1023, off >> 20};
    for (int r = 0; r < nrb; ++r) {
        const double* T[3];
        T[0] = U + (size_t)3 * r * C::USZ + C::SBRA;
        T[1] = T[0] + C::USZ;
        T[2] = T[1] + C::USZ;
        const double I[3] = {T[0][o[0]], T[1][o[1]], T[2][o[2]]};
        double dd[3][3];
#pragma unroll
        for (int x = 0; x < 3; ++x) rys_raw_d1<C>(T[x], o[x], (ex >> (6 * x)) & 63, e2, dd[x][0], dd[x][1], dd[x][2]);
#pragma unroll
        for (int g = 0; g < C::GG; ++g) {
            const int b = b0 + g;
            if (b >= 9) break;
            const int X = b / 3, i = b - 3 * X;
            const double other = i == 0 ? I[1] * I[2] : (i == 1 ? I[0] * I[2] : I[0] * I[1]);
            acc[g] = fma(dd[i][X], other, acc[g]);
        }
    }
}

// Hessian-vector kind: h[3Y + i] += gam * sum_r [(dY V)_i prod_{j != i} I_j +
// (dY I)_i sum_{j != i} V_j prod_{k != i, j} I_k].
template <class C>
QX_HD inline void rys_prod_hvp(const double* O, int nrb, int off, double gam, double* h) {
    const int o[3] = {off & 1023, (off >> 10) & 1023, off >> 20};
    constexpr int S = C::SZ0;
    for (int r = 0; r < nrb; ++r) {
        const double* T[3];
        T[0] = O + (size_t)3 * r * C::UOPS;
        T[1] = T[0] + C::UOPS;
        T[2] = T[1] + C::UOPS;
        double I[3], V[3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            I[x] = T[x][o[x]];
            V[x] = T[x][4 * S + o[x]];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int j = (i + 1) % 3, k = (i + 2) % 3;
            const double P = gam * I[j] * I[k];
            const double Qv = gam * (V[j] * I[k] + I[j] * V[k]);
#pragma unroll
            for (int Y = 0; Y < 3; ++Y)
                h[3 * Y + i] += T[i][(5 + Y) * S + o[i]] * P + T[i][(1 + Y) * S + o[i]] * Qv;
        }
    }
}

// Derivative-tensor kind: the batch's product for op triple (packed 8 bits per
// direction) of component offsets `off`.
template <class C>
QX_HD inline double rys_prod_derk(const double* O, int nrb, int off, int ops) {
    const int ox = off & 1023, oy = (off >> 10) & 1023, oz = off >> 20;
    const int px = (ops & 255) * C::SZ0 + ox, py = ((ops >> 8) & 255) * C::SZ0 + oy,
              pz = ((ops >> 16) & 255) * C::SZ0 + oz;
    double s = 0.0;
    for (int r = 0; r < nrb; ++r) {
        const double* X = O + (size_t)3 * r * C::UOPS;
        s = fma(X[px] * X[C::UOPS + py], X[2 * C::UOPS + pz], s);
    }
    return s;
}

// Multi-index bookkeeping of one derivative tensor element set: the m-th
// non-decreasing k-tuple over the 12 centre-directions (3 * centre + xyz) ->
// per-direction op ranks (packed), the reference's slot (rank of the sorted
// nuclear indices 3 * atom + xyz over M = 3N) and the chain-rule multiplicity
// (ordered picks of centres that give this multiset).  Returns false when the
// tuple does not contribute to the requested slice.
QX_HD inline bool rys_derk_index(int k, long long m, const int* atoms, int M, const int* slice_nu, int slice_k,
                                 int& ops, long long& slot, double& mult) {
    int e[4];
    rys_multiset_unrank(m, k, 12, e);
    int cnt[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    int nu[4];
    for (int i = 0; i < k; ++i) {
        const int c = e[i] / 3, x = e[i] % 3;
        cnt[x][c]++;
        nu[i] = 3 * atoms[c] + x;
    }
    ops = 0;
    for (int x = 0; x < 3; ++x) ops |= rys_op_rank(k, cnt[x][0], cnt[x][1], cnt[x][2], cnt[x][3]) << (8 * x);
    // multiplicity: for each group of equal nuclear indices, (group size)! over
    // the product of (count)! of each distinct centre-direction in the group
    double mlt = 1.0;
    bool used[4] = {false, false, false, false};
    for (int i = 0; i < k; ++i) {
        if (used[i]) continue;
        int members[4], nm = 0;
        for (int j = i; j < k; ++j)
            if (!used[j] && nu[j] == nu[i]) {
                members[nm++] = e[j];
                used[j] = true;
            }
        double num = 1.0, den = 1.0;
        for (int f = 2; f <= nm; ++f) num *= f;
        for (int x = 0; x < nm; ++x) {
            bool first = true;
            for (int y = 0; y < x; ++y)
                if (members[y] == members[x]) first = false;
            if (!first) continue;
            int c = 0;
            for (int y = 0; y < nm; ++y)
                if (members[y] == members[x]) ++c;
            for (int f = 2; f <= c; ++f) den *= f;
        }
        mlt *= num / den;
    }
    mult = mlt;
    // sort nu
    for (int i = 1; i < k; ++i)
        for (int j = i; j > 0 && nu[j - 1] > nu[j]; --j) {
            const int t = nu[j];
            nu[j] = nu[j - 1];
            nu[j - 1] = t;
        }
    if (slice_k) {
        for (int i = 0; i < k; ++i)
            if (nu[i] != slice_nu[i]) return false;
        slot = 0;
        return true;
    }
    slot = rys_multiset_rank(nu, k, M);
    return true;
}

#ifdef __CUDACC__
// ------------------------------------------------------------------ device ---
template <int TS, int TPB>
__device__ __forceinline__ void rys_team_sync(int team) {
    if constexpr (TS == 32) {
        __syncwarp();
    } else if constexpr (TPB == 1) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(TS) : "memory");
    }
}

// Sum of v over the team into thread 0's return value (red: >= TS/32 doubles).
template <int TS, int TPB>
__device__ __forceinline__ double rys_team_sum(double v, double* red, int tid, int team) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if constexpr (TS == 32) {
        return v;
    } else {
        rys_team_sync<TS, TPB>(team);
        if ((tid & 31) == 0) red[tid >> 5] = v;
        rys_team_sync<TS, TPB>(team);
        double s = 0.0;
        if (tid == 0)
            for (int w = 0; w < TS / 32; ++w) s += red[w];
        return s;
    }
}

template <int TS, int TPB>
__device__ __forceinline__ double rys_team_max(double v, double* red, int tid, int team) {
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if constexpr (TS == 32) {
        return v;
    } else {
        rys_team_sync<TS, TPB>(team);
        if ((tid & 31) == 0) red[tid >> 5] = v;
        rys_team_sync<TS, TPB>(team);
        double s = 0.0;
        if (tid == 0)
            for (int w = 0; w < TS / 32; ++w) s = fmax(s, red[w]);
        return s;
    }
}

// Per primitive quartet: nodes/weights, then per root batch the tables and the
// caller's product step `prod(nrb, e2)` (e2: twice the four exponents).
template <class C, int KIND, int LA, int LB, int LC, int LD, class Prod>
__device__ __forceinline__ void rys_primitive(const RysArgs& ra, const PrimPair& p, const PrimPair& r,
                                              const PairInfo& P, const PairInfo& Q, double* uw, double* U, double* O,
                                              const double* w9, int tid, int team, Prod&& prod) {
    RysPrim s;
    rys_prim(p, r, P, Q, s);
    if (tid < 2 * C::NR) uw[tid] = rys_fn<C::NR>(ra.rys, tid, s.T) * (tid >= C::NR ? s.pref : 1.0);
    rys_team_sync<C::TS, C::TPB>(team);
    for (int rb0 = 0; rb0 < C::NR; rb0 += C::RB) {
        const int nrb = C::NR - rb0 < C::RB ? C::NR - rb0 : C::RB;
        if (rb0) rys_team_sync<C::TS, C::TPB>(team);  // the previous batch's products are done
        if constexpr (C::SEQ) {
            rys_phase_units<C>(s, uw, rb0, nrb, U, tid, C::TS);
            rys_team_sync<C::TS, C::TPB>(team);
        } else {
            rys_phase_2d<C>(s, uw, rb0, nrb, U, tid, C::TS);
            rys_team_sync<C::TS, C::TPB>(team);
            for (int b = 1; b < C::B1; ++b) {
                rys_phase_bra<C>(s, b, nrb, U, tid, C::TS);
                rys_team_sync<C::TS, C::TPB>(team);
            }
            for (int d = 0; d < C::D1; ++d) {
                rys_phase_ket<C>(s, d, nrb, U, tid, C::TS);
                rys_team_sync<C::TS, C::TPB>(team);
            }
        }
        if constexpr (C::NOPS > 0) {
            rys_phase_ops<C, KIND, LA, LB, LC, LD>(s, nrb, U, O, w9, tid, C::TS);
            rys_team_sync<C::TS, C::TPB>(team);
        }
        prod(nrb, s.e2);
    }
    rys_team_sync<C::TS, C::TPB>(team);  // products done before the next nodes overwrite
}

template <int LA, int LB, int LC, int LD, int KIND>
__global__ void __launch_bounds__(RysCls<LA, LB, LC, LD, KIND>::BS, RysCls<LA, LB, LC, LD, KIND>::MINB)
    k_rys(RysArgs ra, int mode, long long nwork) {
    using C = RysCls<LA, LB, LC, LD, KIND>;
    constexpr int TS = C::TS, TPB = C::TPB, NCPT = C::NCPT;
    extern __shared__ double rys_sm[];
    const int team = threadIdx.x / TS, tid = threadIdx.x - team * TS;
    double* S = rys_sm + (size_t)team * C::TEAM_SMEM;
    double* uw = S;             // 2 NR nodes/weights
    double* red = S + 32;       // reductions (<= 80)
    double* U = S + C::HDR;     // transfer tables
    double* O = U + (size_t)C::RB * 3 * C::USZ;  // op tables
    int* mops = reinterpret_cast<int*>(S + RYS_HDR);                // RK_DERk: packed ops per multi-index
    long long* mslot = reinterpret_cast<long long*>(S + RYS_HDR + RYS_CHMAX);
    double* mmult = S + RYS_HDR + 2 * RYS_CHMAX;
    const EriArgs& a = ra.e;
    const long long n = a.n;
    const long long nteams = (long long)gridDim.x * TPB;
    for (long long w = (long long)blockIdx.x * TPB + team; w < nwork; w += nteams) {
        long long qi = w;
        int ch = 0;
        if constexpr (KIND >= RK_DER1) {
            qi = w / ra.nchunk;
            ch = (int)(w - qi * ra.nchunk);
        }
        const int2 pq = a.quartets[qi];
        const PairInfo P = a.pairs[pq.x];
        const PairInfo Q = a.pairs[pq.y];
        const int atoms[4] = {P.atom1, P.atom2, Q.atom1, Q.atom2};
        const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
        if constexpr (KIND == RK_PLAIN) {
            if (mode == RMODE_JK && jk_screened(a, pq, P, Q)) continue;  // team-uniform
        } else {
            if (atoms[0] == atoms[1] && atoms[0] == atoms[2] && atoms[0] == atoms[3]) continue;
        }
        // derivative tensors: the work item's multi-indices
        int nm = 0;
        if constexpr (KIND >= RK_DER1) {
            constexpr int k = C::K::ORD;
            const long long ntot = rys_binom(12 + k - 1, k);
            const long long m0 = (long long)ch * ra.chunk;
            nm = (int)((ntot - m0) < ra.chunk ? (ntot - m0) : ra.chunk);
            if (ra.slice_k) {  // slices: skip quartets lacking a requested atom
                bool ok = true;
                for (int i = 0; i < k; ++i) {
                    const int at = ra.slice_nu[i] / 3;
                    if (at != atoms[0] && at != atoms[1] && at != atoms[2] && at != atoms[3]) ok = false;
                }
                if (!ok) continue;
            }
            rys_team_sync<TS, TPB>(team);  // previous work item's epilogue read these
            for (int i = tid; i < nm; i += TS) {
                int ops;
                long long slot;
                double mult;
                const bool keep = rys_derk_index(k, m0 + i, atoms, ra.M, ra.slice_nu, ra.slice_k, ops, slot, mult);
                mops[i] = ops;
                mslot[i] = slot;
                mmult[i] = keep ? mult : 0.0;
            }
            rys_team_sync<TS, TPB>(team);
        }
        // components of this thread
        int offs[NCPT];
        int exps[NCPT];
        double gam[NCPT];
#pragma unroll
        for (int j = 0; j < NCPT; ++j) {
            const int kc = tid + j * TS;
            offs[j] = kc < C::NCOMP ? rys_comp_offsets<C, LA, LB, LC, LD, C::RAW>(kc) : 0;
            if constexpr (rys_is_grad(KIND) || KIND == RK_GRADT)
                exps[j] = kc < C::NCOMP ? rys_comp_exps<C, LA, LB, LC, LD>(kc) : 0;
            gam[j] = 0.0;
            if constexpr (rys_is_grad(KIND) || KIND == RK_HVP) {
                if (kc < C::NCOMP) {
                    const int id = kc % C::ND, ic = (kc / C::ND) % C::NC, ib = (kc / (C::ND * C::NC)) % C::NB,
                              ia = kc / (C::ND * C::NC * C::NB);
                    const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
                    const double* __restrict__ Dm = ra.D;
                    const double fJ = (1.0 + sPQ) * (1.0 + s12) * (1.0 + s34), fK = 1.0 + sPQ;
                    const double kd = 1.0 + (double)(s12 && s34), kx = (double)s12 + (double)s34;
                    gam[j] = ra.cj * fJ * __ldg(Dm + ii * n + jj) * __ldg(Dm + kk * n + ll) +
                             ra.ck * fK * (__ldg(Dm + ii * n + kk) * __ldg(Dm + jj * n + ll) * kd +
                                           __ldg(Dm + ii * n + ll) * __ldg(Dm + jj * n + kk) * kx);
                }
            }
        }
        double w9[9];
        if constexpr (KIND == RK_HVP) {
            bool still = true;
#pragma unroll
            for (int b = 0; b < 9; ++b) {
                w9[b] = __ldg(ra.dir + 3 * atoms[b / 3] + b % 3) - __ldg(ra.dir + 3 * atoms[3] + b % 3);
                still = still && w9[b] == 0.0;
            }
            // the four atoms move alike along the direction: every term is linear
            // in w, so the quartet adds nothing (team-uniform: one quartet per team)
            if (still) continue;
        }
        const int nk = Q.nprim, ntot = P.nprim * nk;
        if constexpr (KIND == RK_PLAIN) {
            double acc[NCPT];
#pragma unroll
            for (int j = 0; j < NCPT; ++j) acc[j] = 0.0;
            for (int t = 0; t < ntot; ++t) {
                const int i = t / nk, jj = t - i * nk;
                rys_primitive<C, KIND, LA, LB, LC, LD>(ra, a.prims[P.prim_off + i], a.prims[Q.prim_off + jj], P, Q,
                                                        uw, U, O, w9, tid, team, [&](int nrb, const double*) {
#pragma unroll
                    for (int j = 0; j < NCPT; ++j)
                        if (tid + j * TS < C::NCOMP) acc[j] += rys_prod_plain<C>(U, nrb, offs[j]);
                });
            }
            if (mode == RMODE_SCHWARZ) {
                double mx = 0.0;
#pragma unroll
                for (int j = 0; j < NCPT; ++j) {
                    const int kc = tid + j * TS;
                    if (kc < C::NCOMP && kc / (C::NC * C::ND) == kc % (C::NC * C::ND)) mx = fmax(mx, fabs(acc[j]));
                }
                mx = rys_team_max<TS, TPB>(mx, red, tid, team);
                if (tid == 0) a.out[pq.x] = mx;
                continue;
            }
#pragma unroll
            for (int j = 0; j < NCPT; ++j) {
                const int kc = tid + j * TS;
                if (kc >= C::NCOMP) continue;
                if (mode == RMODE_UNIQUE) {
                    a.out[a.base + (long long)kc * a.nq + qi] = acc[j];
                    continue;
                }
                const int id = kc % C::ND, ic = (kc / C::ND) % C::NC, ib = (kc / (C::ND * C::NC)) % C::NB,
                          ia = kc / (C::ND * C::NC * C::NB);
                const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
                if (mode == RMODE_JK)
                    jk_images(a.out, a.out2, a.dens, n, ii, jj, kk, ll, s12, s34, sPQ, acc[j]);
                else
                    dense_images(a.out, n, ii, jj, kk, ll, s12, s34, sPQ, acc[j]);
            }
        } else if constexpr (KIND == RK_GRADT) {
            // the first-derivative integrals of the quartet, summed over primitives in
            // registers (GG coordinates per pass), then added into the tile: centre X's
            // block to its atom's rows, minus the sum to the D centre's atom
            constexpr int GG = C::GG;
            for (int b0 = 0; b0 < 9; b0 += GG) {
                double acc[NCPT][GG];
#pragma unroll
                for (int j = 0; j < NCPT; ++j)
#pragma unroll
                    for (int g = 0; g < GG; ++g) acc[j][g] = 0.0;
                for (int t = 0; t < ntot; ++t) {
                    const int i = t / nk, jj = t - i * nk;
                    rys_primitive<C, KIND, LA, LB, LC, LD>(ra, a.prims[P.prim_off + i], a.prims[Q.prim_off + jj], P,
                                                            Q, uw, U, O, w9, tid, team, [&](int nrb, const double* e2) {
#pragma unroll
                        for (int j = 0; j < NCPT; ++j)
                            if (tid + j * TS < C::NCOMP)
                                rys_prod_gradt<C>(U, nrb, offs[j], exps[j], e2, b0, acc[j]);
                    });
                }
#pragma unroll
                for (int j = 0; j < NCPT; ++j) {
                    const int kc = tid + j * TS;
                    if (kc >= C::NCOMP) continue;
                    const long long e = qi * C::NCOMP + kc;
#pragma unroll
                    for (int g = 0; g < GG; ++g) {
                        const int b = b0 + g;
                        if (b >= 9) break;
                        const int X = b / 3, x = b - 3 * X;
                        tile_add(a.out, ra.tile_E, 3 * atoms[X] + x, e, ra.tile_images, s12, s34, sPQ, acc[j][g]);
                        tile_add(a.out, ra.tile_E, 3 * atoms[3] + x, e, ra.tile_images, s12, s34, sPQ, -acc[j][g]);
                    }
                }
            }
        } else if constexpr (rys_is_grad(KIND) || KIND == RK_HVP) {
            double g[9];
#pragma unroll
            for (int b = 0; b < 9; ++b) g[b] = 0.0;
            for (int t = 0; t < ntot; ++t) {
                const int i = t / nk, jj = t - i * nk;
                rys_primitive<C, KIND, LA, LB, LC, LD>(ra, a.prims[P.prim_off + i], a.prims[Q.prim_off + jj], P, Q,
                                                        uw, U, O, w9, tid, team, [&](int nrb, const double* e2) {
#pragma unroll
                    for (int j = 0; j < NCPT; ++j)
                        if (tid + j * TS < C::NCOMP) {
                            if constexpr (rys_is_grad(KIND))
                                rys_prod_grad<C>(U, nrb, offs[j], exps[j], e2, gam[j], g);
                            else
                                rys_prod_hvp<C>(O, nrb, offs[j], gam[j], g);
                        }
                });
            }
#pragma unroll
            for (int b = 0; b < 9; ++b) g[b] = rys_team_sum<TS, TPB>(g[b], red + 8 * (b % 8), tid, team);
            if (tid == 0) {
                for (int x = 0; x < 3; ++x) {
                    atomicAdd(ra.grad + 3 * atoms[0] + x, g[x]);
                    atomicAdd(ra.grad + 3 * atoms[1] + x, g[3 + x]);
                    atomicAdd(ra.grad + 3 * atoms[2] + x, g[6 + x]);
                    atomicAdd(ra.grad + 3 * atoms[3] + x, -(g[x] + g[3 + x] + g[6 + x]));
                }
            }
        } else {
            // derivative tensors: nm multi-indices x NCPT components
            constexpr int MG = C::MG;
            double acc[NCPT][MG];
            const long long n4 = n * n * n * n;
            for (int m0 = 0; m0 < nm; m0 += MG) {
                const int mn = nm - m0 < MG ? nm - m0 : MG;
#pragma unroll
                for (int j = 0; j < NCPT; ++j)
#pragma unroll
                    for (int mm = 0; mm < MG; ++mm) acc[j][mm] = 0.0;
                for (int t = 0; t < ntot; ++t) {
                    const int i = t / nk, jj = t - i * nk;
                    rys_primitive<C, KIND, LA, LB, LC, LD>(ra, a.prims[P.prim_off + i], a.prims[Q.prim_off + jj], P,
                                                            Q, uw, U, O, w9, tid, team, [&](int nrb, const double*) {
#pragma unroll
                        for (int j = 0; j < NCPT; ++j)
                            if (tid + j * TS < C::NCOMP)
#pragma unroll
                                for (int mm = 0; mm < MG; ++mm)
                                    if (mm < mn) acc[j][mm] += rys_prod_derk<C>(O, nrb, offs[j], mops[m0 + mm]);
                    });
                }
#pragma unroll
                for (int j = 0; j < NCPT; ++j) {
                    const int kc = tid + j * TS;
                    if (kc >= C::NCOMP) continue;
                    const int id = kc % C::ND, ic = (kc / C::ND) % C::NC, ib = (kc / (C::ND * C::NC)) % C::NB,
                              ia = kc / (C::ND * C::NC * C::NB);
                    const long long ii = P.bf1 + ia, jj = P.bf2 + ib, kk = Q.bf1 + ic, ll = Q.bf2 + id;
                    for (int mm = 0; mm < mn; ++mm) {
                        const double mult = mmult[m0 + mm];
                        if (mult == 0.0) continue;
                        if (ra.tile_E)  // order 1: the slot is the nuclear index
                            tile_add(a.out, ra.tile_E, (int)mslot[m0 + mm], qi * C::NCOMP + kc, ra.tile_images, s12,
                                     s34, sPQ, mult * acc[j][mm]);
                        else
                            atomic_images_w(a.out + mslot[m0 + mm] * n4, n, ii, jj, kk, ll, s12, s34, sPQ,
                                            mult * acc[j][mm]);
                    }
                }
            }
        }
    }
}

// Host launcher of one class and kind; returns false when the class's tables do
// not fit shared memory for this kind.
template <int LA, int LB, int LC, int LD, int KIND>
bool launch_rys(const RysArgs& ra, int mode, long long nwork, cudaStream_t s) {
    using C = RysCls<LA, LB, LC, LD, KIND>;
    if constexpr (!C::FITS) {
        return false;
    } else {
        if (nwork <= 0) return true;
        auto k = k_rys<LA, LB, LC, LD, KIND>;
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
            attr = true;
        }
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, C::BS, C::SMEM);
        if (per_sm < 1) per_sm = 1;
        long long nb = (nwork + C::TPB - 1) / C::TPB;
        const long long cap = 148LL * per_sm * 8;
        if (nb > cap) nb = cap;
        k<<<(unsigned)nb, C::BS, C::SMEM, s>>>(ra, mode, nwork);
        return true;
    }
}
#endif  // __CUDACC__

}  // namespace qx
