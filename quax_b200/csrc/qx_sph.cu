// qx_sph.cu -- Cartesian -> real-solid-harmonic transform of unique ERI blocks.
//
// A class's unique layout holds, per Cartesian component (ka, kb, kc, kd), one
// contiguous plane of nq values (one per screened quartet).  Each spherical
// component (sa, sb, sc, sd) is a short linear combination of those planes:
//   out[sa,sb,sc,sd][q] = sum T_a[sa,ka] T_b[sb,kb] T_c[sc,kc] T_d[sd,kd] in[ka,kb,kc,kd][q]
// with the per-shell matrices T_l (2l+1, ncart(l)), of which each row has 1-4
// non-zero entries.  One thread per output value walks the non-zero entries, so
// every read and write is coalesced across the quartets of a warp and the input
// planes, a few MB per class, are re-read from L2.  The Python layer passes the
// matrices (quax_b200/integrals/spherical.py: cart2sph), so the convention lives
// in one place.
#include <cmath>

#include "quax_b200.h"

namespace {

constexpr int kSphLmax = QX_MAX_L;
constexpr int kSphTerms = 128;

// Non-zero entries of T_l, row by row: row m of l spans [start[l][m], start[l][m+1]).
struct SphTab {
    int start[kSphLmax + 1][2 * kSphLmax + 2];
    int cart[kSphTerms];
    double coef[kSphTerms];
};

__global__ void __launch_bounds__(256) k_cart2sph(const double* __restrict__ in, double* __restrict__ out, int la,
                                                  int lb, int lc, int ld, long long nq, SphTab t) {
    const int Sb = 2 * lb + 1, Sc = 2 * lc + 1, Sd = 2 * ld + 1;
    const int NB = (lb + 1) * (lb + 2) / 2, NC = (lc + 1) * (lc + 2) / 2, ND = (ld + 1) * (ld + 2) / 2;
    const long long total = nq * (2 * la + 1) * Sb * Sc * Sd;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long qi = e % nq;
        int ks = (int)(e / nq);
        const int sd = ks % Sd;
        ks /= Sd;
        const int sc = ks % Sc;
        ks /= Sc;
        const int sb = ks % Sb, sa = ks / Sb;
        double v = 0.0;
        for (int ia = t.start[la][sa]; ia < t.start[la][sa + 1]; ++ia)
            for (int ib = t.start[lb][sb]; ib < t.start[lb][sb + 1]; ++ib) {
                const double cab = t.coef[ia] * t.coef[ib];
                const int kab = t.cart[ia] * NB + t.cart[ib];
                for (int ic = t.start[lc][sc]; ic < t.start[lc][sc + 1]; ++ic)
                    for (int id = t.start[ld][sd]; id < t.start[ld][sd + 1]; ++id) {
                        const long long k = ((long long)(kab * NC + t.cart[ic]) * ND + t.cart[id]) * nq + qi;
                        v = fma(cab * t.coef[ic] * t.coef[id], __ldg(in + k), v);
                    }
            }
        out[e] = v;
    }
}

}  // namespace

void qx_set_last_error(const char* msg);  // defined with the other error state

static int sph_fail(int code, const char* msg) {
    qx_set_last_error(msg);  // reported by qx_last_error()
    return code;
}

// Transforms one class's unique Cartesian blocks (in_dev: ncart(la) ncart(lb)
// ncart(lc) ncart(ld) planes of nq doubles) into spherical blocks (out_dev:
// (2la+1)(2lb+1)(2lc+1)(2ld+1) planes of nq doubles, the same element-major
// order).  T_host: the matrices T_l (2l+1, ncart(l)) for l = 0..QX_MAX_L, row-major
// and concatenated (1 + 9 + 30 + 70 doubles).  Allocates nothing; asynchronous on
// `stream`.
extern "C" int qx_cart2sph_block(const double* in_dev, double* out_dev, const int* l4, long long nq,
                                 const double* T_host, void* stream) {
    if (!l4 || !T_host || nq < 0) return sph_fail(QX_E_INVALID, "qx_cart2sph_block: bad argument");
    for (int i = 0; i < 4; ++i)
        if (l4[i] < 0 || l4[i] > kSphLmax) return sph_fail(QX_E_UNSUPPORTED, "qx_cart2sph_block: l out of range");
    if (nq == 0) return QX_OK;
    if (!in_dev || !out_dev) return sph_fail(QX_E_INVALID, "qx_cart2sph_block: null buffer");
    SphTab t{};
    int n = 0;
    const double* T = T_host;
    for (int l = 0; l <= kSphLmax; ++l) {
        const int nc = (l + 1) * (l + 2) / 2;
        for (int m = 0; m < 2 * l + 1; ++m) {
            t.start[l][m] = n;
            for (int k = 0; k < nc; ++k) {
                const double c = T[m * nc + k];
                if (!std::isfinite(c)) return sph_fail(QX_E_INVALID, "qx_cart2sph_block: non-finite coefficient");
                if (c == 0.0) continue;
                if (n == kSphTerms) return sph_fail(QX_E_INVALID, "qx_cart2sph_block: too many coefficients");
                t.cart[n] = k;
                t.coef[n] = c;
                ++n;
            }
        }
        t.start[l][2 * l + 1] = n;
        T += (2 * l + 1) * nc;
    }
    const long long total = nq * (2 * l4[0] + 1) * (2 * l4[1] + 1) * (2 * l4[2] + 1) * (2 * l4[3] + 1);
    long long nb = (total + 255) / 256;
    if (nb > 148LL * 16) nb = 148LL * 16;
    k_cart2sph<<<(unsigned)nb, 256, 0, (cudaStream_t)stream>>>(in_dev, out_dev, l4[0], l4[1], l4[2], l4[3], nq, t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sph_fail(QX_E_CUDA, cudaGetErrorString(e));
    return QX_OK;
}
