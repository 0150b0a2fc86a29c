// Host build of the Rys engine's per-primitive phases (test infrastructure).
//
// The device kernel runs the same functions (qx_rys.cuh: rys_prim, rys_fn, the
// table builders and the product steps) over a team of threads; here one host
// thread runs them with (tid, nth) = (0, 1), so tests on a machine without a GPU
// can compare the engine's arithmetic with the oracle: plain integrals, the nine
// first-derivative sums of the adjoint gradient, the Hessian-vector sums and the
// derivative blocks of orders 1 and 2, with either table build and with the root
// batching of the compiled kernel.
#include <cmath>
#include <vector>

#include "qx_rys.cuh"

using namespace qx;

namespace {

const double g_tab[] = {QX_RYS_TAB_DATA QX_RYS_ASYM_Y_DATA, QX_RYS_ASYM_W_DATA};

struct Sh {
    int l, n;
    const double *c, *e, *w;  // centre (3), exponents, normalised coefficients
};

void make_pair(const Sh& a, const Sh& b, PairInfo& P, std::vector<PrimPair>& pr) {
    const double kfac = std::sqrt(2.0) * std::pow(M_PI, 1.25);
    P.Ax = a.c[0];
    P.Ay = a.c[1];
    P.Az = a.c[2];
    P.ABx = a.c[0] - b.c[0];
    P.ABy = a.c[1] - b.c[1];
    P.ABz = a.c[2] - b.c[2];
    const double AB2 = P.ABx * P.ABx + P.ABy * P.ABy + P.ABz * P.ABz;
    P.nprim = a.n * b.n;
    P.prim_off = 0;
    P.l1 = a.l;
    P.l2 = b.l;
    for (int i = 0; i < a.n; ++i)
        for (int j = 0; j < b.n; ++j) {
            PrimPair r;
            const double x = a.e[i], y = b.e[j];
            r.zeta = x + y;
            r.oo2z = 0.5 / r.zeta;
            r.PAx = -(y / r.zeta) * (a.c[0] - b.c[0]);
            r.PAy = -(y / r.zeta) * (a.c[1] - b.c[1]);
            r.PAz = -(y / r.zeta) * (a.c[2] - b.c[2]);
            r.Px = a.c[0] + r.PAx;
            r.Py = a.c[1] + r.PAy;
            r.Pz = a.c[2] + r.PAz;
            r.K = kfac * a.w[i] * b.w[j] * std::exp(-x * y / r.zeta * AB2) / r.zeta;
            r.alpha = x;
            pr.push_back(r);
        }
}

// build: 0 level-parallel tables, 1 per-unit tables, 2 as the compiled kernel
// (its per-unit/level-parallel choice and its RB-root batches).
template <int LA, int LB, int LC, int LD, int KIND>
void run(const Sh* s, const double* gam, const double* w9, int build, double* out) {
    using C = RysCls<LA, LB, LC, LD, KIND>;
    PairInfo P, Q;
    std::vector<PrimPair> pp, qq;
    make_pair(s[0], s[1], P, pp);
    make_pair(s[2], s[3], Q, qq);
    std::vector<double> uw(2 * C::NR), U((size_t)C::NR * 3 * C::USZ), O((size_t)C::NR * 3 * (C::UOPS + 1));
    // derivative tensors: every multi-index of the quartet's 12 centre-directions
    const int nmulti = KIND >= RK_DER1 ? rys_binom(12 + C::K::ORD - 1, C::K::ORD) : 1;
    std::vector<int> mops(nmulti, 0);
    if constexpr (KIND >= RK_DER1) {
        const int atoms[4] = {0, 1, 2, 3};
        for (int m = 0; m < nmulti; ++m) {
            long long slot;
            double mult;
            rys_derk_index(C::K::ORD, m, atoms, 12, nullptr, 0, mops[m], slot, mult);
        }
    }
    std::vector<double> acc((size_t)C::NCOMP * nmulti, 0.0);
    double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int rb = build == 2 ? C::RB : C::NR;
    const bool seq = build == 1 || (build == 2 && C::SEQ);
    for (const PrimPair& p : pp)
        for (const PrimPair& r : qq) {
            RysPrim st;
            rys_prim(p, r, P, Q, st);
            for (int f = 0; f < 2 * C::NR; ++f) uw[f] = rys_fn<C::NR>(g_tab, f, st.T) * (f >= C::NR ? st.pref : 1.0);
            for (int rb0 = 0; rb0 < C::NR; rb0 += rb) {
                const int nrb = C::NR - rb0 < rb ? C::NR - rb0 : rb;
                if (seq) {
                    rys_phase_units<C>(st, uw.data(), rb0, nrb, U.data(), 0, 1);
                } else {
                    rys_phase_2d<C>(st, uw.data(), rb0, nrb, U.data(), 0, 1);
                    for (int b = 1; b < C::B1; ++b) rys_phase_bra<C>(st, b, nrb, U.data(), 0, 1);
                    for (int d = 0; d < C::D1; ++d) rys_phase_ket<C>(st, d, nrb, U.data(), 0, 1);
                }
                if constexpr (C::NOPS > 0) rys_phase_ops<C, KIND, LA, LB, LC, LD>(st, nrb, U.data(), O.data(), w9, 0, 1);
                for (int kc = 0; kc < C::NCOMP; ++kc) {
                    const int off = rys_comp_offsets<C, LA, LB, LC, LD, C::RAW>(kc);
                    if constexpr (KIND == RK_PLAIN)
                        acc[kc] += rys_prod_plain<C>(U.data(), nrb, off);
                    else if constexpr (KIND == RK_GRAD)
                        rys_prod_grad<C>(U.data(), nrb, off, rys_comp_exps<C, LA, LB, LC, LD>(kc), st.e2, gam[kc], g);
                    else if constexpr (KIND == RK_HVP)
                        rys_prod_hvp<C>(O.data(), nrb, off, gam[kc], g);
                    else
                        for (int m = 0; m < nmulti; ++m)
                            acc[(size_t)m * C::NCOMP + kc] += rys_prod_derk<C>(O.data(), nrb, off, mops[m]);
                }
            }
        }
    if constexpr (KIND == RK_GRAD || KIND == RK_HVP)
        for (int b = 0; b < 9; ++b) out[b] = g[b];
    else
        for (size_t i = 0; i < acc.size(); ++i) out[i] = acc[i];
}

}  // namespace

// The classes this harness covers, in the order of rys_host_class().
static const int kL[][4] = {{0, 0, 0, 0}, {1, 0, 1, 0}, {2, 1, 1, 0}, {3, 0, 0, 0}, {3, 2, 1, 0}, {2, 2, 2, 1},
                            {3, 1, 2, 2}, {3, 3, 2, 0}, {3, 3, 3, 2}, {3, 3, 3, 3}};

extern "C" int rys_host_nclass(void) { return (int)(sizeof kL / sizeof kL[0]); }

extern "C" void rys_host_class(int i, int* l4) {
    for (int k = 0; k < 4; ++k) l4[k] = kL[i][k];
}

// kind 0: plain block (NCOMP values); 1: the nine sums g[3X + x] = sum_kc gam_kc
// d/dX_x (ab|cd)_kc, X = A, B, C; 2: the Hessian-vector sums h[3X + x] = sum_kc
// gam_kc sum_V w9[V] d2/dX_x dV (ab|cd)_kc; 11, 12: the derivative blocks of
// orders 1 and 2, one NCOMP block per sorted multi-index of the 12
// centre-directions 3 * centre + xyz.  Shells: centres cen[12], primitive counts
// np[4], exponents and normalised coefficients concatenated.
extern "C" int rys_host(int kind, int cls, int build, const double* cen, const int* np, const double* exps,
                        const double* wts, const double* gam, const double* w9, double* out) {
    if (cls < 0 || cls >= rys_host_nclass() || build < 0 || build > 2) return -1;
    if (kind != 0 && kind != 1 && kind != 2 && kind != 11 && kind != 12) return -1;
    Sh s[4];
    int o = 0;
    for (int c = 0; c < 4; ++c) {
        s[c].l = kL[cls][c];
        s[c].n = np[c];
        s[c].c = cen + 3 * c;
        s[c].e = exps + o;
        s[c].w = wts + o;
        o += np[c];
    }
#define QX_HOST_CASE(i, a, b, c, d)                                                   \
    case i:                                                                           \
        if (kind == 0) run<a, b, c, d, RK_PLAIN>(s, gam, w9, build, out);             \
        if (kind == 1) run<a, b, c, d, RK_GRAD>(s, gam, w9, build, out);              \
        if (kind == 2) run<a, b, c, d, RK_HVP>(s, gam, w9, build, out);               \
        if (kind == 11) run<a, b, c, d, RK_DER1>(s, gam, w9, build, out);             \
        if (kind == 12) run<a, b, c, d, RK_DER2>(s, gam, w9, build, out);             \
        return 0;
    switch (cls) {
        QX_HOST_CASE(0, 0, 0, 0, 0)
        QX_HOST_CASE(1, 1, 0, 1, 0)
        QX_HOST_CASE(2, 2, 1, 1, 0)
        QX_HOST_CASE(3, 3, 0, 0, 0)
        QX_HOST_CASE(4, 3, 2, 1, 0)
        QX_HOST_CASE(5, 2, 2, 2, 1)
        QX_HOST_CASE(6, 3, 1, 2, 2)
        QX_HOST_CASE(7, 3, 3, 2, 0)
        QX_HOST_CASE(8, 3, 3, 3, 2)
        QX_HOST_CASE(9, 3, 3, 3, 3)
    }
#undef QX_HOST_CASE
    return -1;
}
