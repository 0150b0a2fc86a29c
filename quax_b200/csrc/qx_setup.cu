// qx_setup.cu -- host-side set-up shared by qx_initialize and the no-alloc path.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "quax_b200.h"
#include "qx_setup.h"

namespace qx {

namespace {
int set_err(std::string& err, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
}

double dfact(int n) {
    double r = 1.0;
    while (n > 1) {
        r *= n;
        n -= 2;
    }
    return r;
}
}  // namespace

int normalize_shells(const char* who, int natom, int nshell, const int* shell_l, const int* shell_nprim,
                     const int* shell_atom, const double* exps, const double* coefs, int lmax, ShellTables& t,
                     std::string& err) {
    t = ShellTables();
    int off = 0;
    for (int s = 0; s < nshell; ++s) {
        const int l = shell_l[s], k = shell_nprim[s], at = shell_atom[s];
        if (l < 0 || l > lmax)
            return set_err(err, QX_E_UNSUPPORTED, "%s: shell %d has l=%d (compiled max %d)", who, s, l, lmax);
        if (k <= 0 || k > 64)
            return set_err(err, QX_E_INVALID, "%s: shell %d has %d primitives (1..64 allowed)", who, s, k);
        if (at < 0 || at >= natom) return set_err(err, QX_E_INVALID, "%s: shell %d on atom %d of %d", who, s, at, natom);
        t.l.push_back(l);
        t.nprim.push_back(k);
        t.atom.push_back(at);
        t.poff.push_back(off);
        t.bf.push_back(t.nbf);
        const double df = dfact(2 * l - 1);
        std::vector<double> c(k);
        for (int p = 0; p < k; ++p) {
            const double a = exps[off + p];
            if (!(a > 0.0) || !std::isfinite(a) || !std::isfinite(coefs[off + p]))
                return set_err(err, QX_E_INVALID, "%s: shell %d primitive %d has exponent %g", who, s, p, a);
            c[p] = coefs[off + p] * std::sqrt(std::pow(2.0, l) * std::pow(2.0 * a, l + 1.5) / (std::pow(M_PI, 1.5) * df));
        }
        double nrm = 0.0;
        for (int p = 0; p < k; ++p)
            for (int q = 0; q < k; ++q)
                nrm += c[p] * c[q] * df * std::pow(M_PI, 1.5) /
                       (std::pow(2.0, l) * std::pow(exps[off + p] + exps[off + q], l + 1.5));
        if (!(nrm > 0.0)) return set_err(err, QX_E_INVALID, "%s: shell %d has a degenerate contraction", who, s);
        for (int p = 0; p < k; ++p) {
            t.alpha.push_back(exps[off + p]);
            t.coef.push_back(c[p] / std::sqrt(nrm));
        }
        off += k;
        t.nbf += (l + 1) * (l + 2) / 2;
    }
    return QX_OK;
}

void build_pairs(const ShellTables& t, const double* coords, std::vector<PrimPair>& prims,
                 std::vector<PairInfo>& pairs, std::vector<int>& pcls) {
    const int nshell = (int)t.l.size();
    const double kfac = std::sqrt(2.0) * std::pow(M_PI, 1.25);
    prims.clear();
    pairs.clear();
    pcls.clear();
    for (int s1 = 0; s1 < nshell; ++s1)
        for (int s2 = 0; s2 <= s1; ++s2) {
            int f = s1, g = s2;
            if (t.l[s2] > t.l[s1]) std::swap(f, g);
            const double* A = coords + 3 * t.atom[f];
            const double* B = coords + 3 * t.atom[g];
            PairInfo pi;
            pi.Ax = A[0]; pi.Ay = A[1]; pi.Az = A[2];
            pi.ABx = A[0] - B[0]; pi.ABy = A[1] - B[1]; pi.ABz = A[2] - B[2];
            const double AB2 = pi.ABx * pi.ABx + pi.ABy * pi.ABy + pi.ABz * pi.ABz;
            pi.prim_off = (int)prims.size();
            pi.nprim = t.nprim[f] * t.nprim[g];
            pi.bf1 = t.bf[f]; pi.bf2 = t.bf[g];
            pi.s1 = f; pi.s2 = g;
            pi.atom1 = t.atom[f]; pi.atom2 = t.atom[g];
            pi.l1 = t.l[f]; pi.l2 = t.l[g];
            for (int p = 0; p < t.nprim[f]; ++p)
                for (int q = 0; q < t.nprim[g]; ++q) {
                    const double a = t.alpha[t.poff[f] + p], b = t.alpha[t.poff[g] + q];
                    const double ca = t.coef[t.poff[f] + p], cb = t.coef[t.poff[g] + q];
                    PrimPair r;
                    r.zeta = a + b;
                    r.oo2z = 0.5 / r.zeta;
                    // P - A = -(b / zeta)(A - B), exactly zero for a one-centre pair
                    // (forming P first and subtracting A leaves ~1e-15 there, which
                    // tight exponents amplify beyond 1e-12 in integrals that vanish
                    // by symmetry)
                    r.PAx = -(b / r.zeta) * (A[0] - B[0]);
                    r.PAy = -(b / r.zeta) * (A[1] - B[1]);
                    r.PAz = -(b / r.zeta) * (A[2] - B[2]);
                    r.Px = A[0] + r.PAx; r.Py = A[1] + r.PAy; r.Pz = A[2] + r.PAz;
                    r.K = kfac * ca * cb * std::exp(-a * b / r.zeta * AB2) / r.zeta;
                    r.alpha = a;
                    prims.push_back(r);
                }
            pairs.push_back(pi);
            pcls.push_back(pi.l1 * (pi.l1 + 1) / 2 + pi.l2);
        }
}

// F_m on the grid T_g = g / BOYS_INV_H: the series for the top order in
// extended precision, then the downward recursion F_m = (2T F_{m+1} + e^{-T}) /
// (2m + 1) (Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory,
// sec. 9.8).
const std::vector<double>& boys_table() {
    static std::once_flag once;
    static std::vector<double> tab;
    std::call_once(once, [] {
        tab.assign((size_t)BOYS_NG * BOYS_NM, 0.0);
        for (int g = 0; g < BOYS_NG; ++g) {
            const double T = g / BOYS_INV_H;
            double F[BOYS_NM];
            const int M = BOYS_NM - 1;
            if (T == 0.0) {
                for (int m = 0; m <= M; ++m) F[m] = 1.0 / (2 * m + 1);
            } else {
                long double term = 1.0L / (2 * M + 1), sum = term;
                for (int k = 1; k < 4000; ++k) {
                    term *= 2.0L * T / (2 * M + 2 * k + 1);
                    sum += term;
                    if (term < sum * 1e-21L) break;
                }
                const long double eT = expl(-(long double)T);
                long double Fm = eT * sum;
                F[M] = (double)Fm;
                for (int m = M; m > 0; --m) {
                    Fm = (2.0L * T * Fm + eT) / (2 * m - 1);
                    F[m - 1] = (double)Fm;
                }
            }
            for (int m = 0; m < BOYS_NM; ++m) tab[(size_t)g * BOYS_NM + m] = F[m];
        }
    });
    return tab;
}

}  // namespace qx
