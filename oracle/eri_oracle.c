/*
 * eri_oracle.c -- CPU FP64 oracle for the two-electron integral path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load this library, and only as the results to
 * compare with (or the timed CPU arm).  The product path never calls it.
 *
 * What it restates:
 *   - Schwarz screening with the reference's semantics
 *       quax/integrals/libint_interface.cc:158-229  (K_ab = max |(f1 f2|f1 f2)|,
 *       not square-rooted; pair kept iff K_ab >= thr^2 / max K; quartet skipped
 *       iff K_ab * K_cd < thr^2, libint_interface.cc:555,2638)
 *   - the dense ERI tensor, row-major i*n^3+j*n^2+k*n+l, bra pairs x all ket
 *       pairs with the 4-permutation scatter, libint_interface.cc:486-647
 *   - the first-derivative tensor (3N, n, n, n, n), nuclear index
 *       (atom, xyz) = sum over shells on that atom of Libint buffer 3*shell+xyz,
 *       quartets on a single atom skipped, libint_interface.cc:2582-2779
 *   - one derivative slice for a deriv_vec, libint_interface.cc:1097-1335
 *   - index helpers quax/integrals/utils.h:95-174
 * The arithmetic itself lives in the third-party, un-vendored Libint2 (conda-forge
 * "libint", version unpinned by the reference, devtools/conda-envs/test_env.yaml:6).
 * It is restated here from the published method Libint implements:
 *   Obara & Saika, J. Chem. Phys. 84, 3963 (1986) -- vertical recurrence (VRR);
 *   Head-Gordon & Pople, J. Chem. Phys. 89, 5777 (1988) -- horizontal recurrence
 *   (HRR) applied to contracted integrals;
 *   Gaussian derivative identity d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}.
 * Boys function: power series F_m(T) = e^{-T} sum_k (2T)^k / prod_{i=0..k}(2m+2i+1)
 * at the top order followed by downward recursion, and erf + upward recursion for
 * large T (Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory, 9.8).
 *
 * Parity status: the reference's integral values come from Libint, which cannot be
 * built or imported here, and the reference stores no golden integral vectors (its
 * tests compare against psi4 at run time).  Integral values are therefore pinned
 * by closed forms, published textbook values (Szabo & Ostlund H2/STO-3G) and an
 * independent McMurchie-Davidson implementation (oracle/md_check.py); parity with
 * Libint itself is unpinned.  The integer bookkeeping is pinned against the
 * reference's own utils.h compiled from source (oracle/ref_utils_shim.cpp).
 *
 * Conventions: Libint "standard" Cartesian ordering (xx,xy,xz,yy,yz,zz,...);
 * Libint normalisation (x^l component of the contracted shell has unit norm).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define QXO_LMAX 28 /* highest AM in any intermediate */

static inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static inline int hoff(int l) { return l * (l + 1) * (l + 2) / 6; }
/* global index of Cartesian component (lx,ly,lz) in the concatenation over l */
static inline int cidx(int lx, int ly, int lz) {
    int l = lx + ly + lz, k = l - lx;
    return hoff(l) + k * (k + 1) / 2 + lz;
}
/* local index inside AM l */
static inline int lidx(int lx, int ly, int lz) {
    int k = ly + lz;
    (void)lx;
    return k * (k + 1) / 2 + lz;
}

static int g_comp[QXO_LMAX + 2][((QXO_LMAX + 2) * (QXO_LMAX + 3)) / 2][3];
static int g_tables_ready = 0;

static void init_tables(void) {
    if (g_tables_ready) return;
    for (int l = 0; l <= QXO_LMAX + 1; ++l) {
        int i = 0;
        for (int lx = l; lx >= 0; --lx)
            for (int ly = l - lx; ly >= 0; --ly) {
                g_comp[l][i][0] = lx;
                g_comp[l][i][1] = ly;
                g_comp[l][i][2] = l - lx - ly;
                ++i;
            }
    }
    g_tables_ready = 1;
}

/* ------------------------------------------------------------------ basis ---- */
typedef struct {
    int nshell, natom;
    const int *l, *nprim, *atom, *prim_off;
    const double *center; /* nshell*3, bohr */
    const double *alpha;  /* exponents */
    const double *coef;   /* normalised coefficients (see qxo_normalize) */
} qxo_basis;

static double dfact(int n) {
    double r = 1.0;
    while (n > 1) { r *= n; n -= 2; }
    return r;
}

/* Libint-convention normalisation: primitive norm of x^l, then unit self-overlap
 * of the contracted x^l component. */
int qxo_normalize(int l, int nprim, const double *alpha, const double *c_in, double *c_out) {
    double df = dfact(2 * l - 1);
    for (int p = 0; p < nprim; ++p) {
        double a = alpha[p];
        if (!(a > 0.0)) return -1;
        c_out[p] = c_in[p] * sqrt(pow(2.0, l) * pow(2.0 * a, l + 1.5) / (pow(M_PI, 1.5) * df));
    }
    double s = 0.0;
    for (int p = 0; p < nprim; ++p)
        for (int q = 0; q < nprim; ++q)
            s += c_out[p] * c_out[q] * df * pow(M_PI, 1.5) / (pow(2.0, l) * pow(alpha[p] + alpha[q], l + 1.5));
    if (!(s > 0.0)) return -1;
    s = 1.0 / sqrt(s);
    for (int p = 0; p < nprim; ++p) c_out[p] *= s;
    return 0;
}

/* ------------------------------------------------------------------ Boys ----- */
void qxo_boys(int mmax, double T, double *F) {
    if (T < 1e-300) {
        for (int m = 0; m <= mmax; ++m) F[m] = 1.0 / (2 * m + 1);
        return;
    }
    double eT = exp(-T);
    if (T < 45.0) {
        /* series at the top order, then downward recursion (stable) */
        double term = 1.0 / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 2000; ++k) {
            term *= 2.0 * T / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-18) break;
        }
        F[mmax] = eT * sum;
        for (int m = mmax; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + eT) / (2 * m - 1);
    } else {
        F[0] = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
        for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - eT) / (2.0 * T);
    }
}

/* ------------------------------------------------------------------ VRR ------ */
/* Obara-Saika VRR for [e0|f0]^(m), 0<=e<=E, 0<=f<=F, 0<=m<=E+F-e-f.
 * v is [hoff(E+1)][hoff(F+1)][E+F+1]. */
static void vrr(int E, int F, double zeta, double eta, const double PA[3], const double WP[3],
                const double QC[3], const double WQ[3], double rho, const double *Fm, double pref,
                double *v) {
    const int NF = hoff(F + 1), M = E + F + 1;
#define V(eh, fh, m) v[((size_t)(eh) * NF + (fh)) * M + (m)]
    for (int m = 0; m <= E + F; ++m) V(0, 0, m) = pref * Fm[m];
    const double oo2z = 0.5 / zeta, roz = rho / zeta, oo2e = 0.5 / eta, roe = rho / eta;
    const double oo2ze = 0.5 / (zeta + eta);
    for (int e = 1; e <= E; ++e) {
        for (int c = 0; c < ncart(e); ++c) {
            const int *x = g_comp[e][c];
            int i = x[0] > 0 ? 0 : (x[1] > 0 ? 1 : 2);
            int n = x[i];
            int y[3] = {x[0], x[1], x[2]};
            y[i] -= 1;
            int hm = cidx(y[0], y[1], y[2]);
            int hmm = -1;
            if (n >= 2) { y[i] -= 1; hmm = cidx(y[0], y[1], y[2]); }
            int h = hoff(e) + c;
            for (int m = 0; m <= E + F - e; ++m) {
                double r = PA[i] * V(hm, 0, m) + WP[i] * V(hm, 0, m + 1);
                if (hmm >= 0) r += (n - 1) * oo2z * (V(hmm, 0, m) - roz * V(hmm, 0, m + 1));
                V(h, 0, m) = r;
            }
        }
    }
    for (int f = 1; f <= F; ++f) {
        for (int c = 0; c < ncart(f); ++c) {
            const int *x = g_comp[f][c];
            int j = x[0] > 0 ? 0 : (x[1] > 0 ? 1 : 2);
            int nf = x[j];
            int y[3] = {x[0], x[1], x[2]};
            y[j] -= 1;
            int gm = cidx(y[0], y[1], y[2]);
            int gmm = -1;
            if (nf >= 2) { y[j] -= 1; gmm = cidx(y[0], y[1], y[2]); }
            int g = hoff(f) + c;
            for (int e = 0; e <= E; ++e) {
                for (int ce = 0; ce < ncart(e); ++ce) {
                    const int *xe = g_comp[e][ce];
                    int ne = xe[j];
                    int h = hoff(e) + ce;
                    int hm = -1;
                    if (ne >= 1) {
                        int z[3] = {xe[0], xe[1], xe[2]};
                        z[j] -= 1;
                        hm = cidx(z[0], z[1], z[2]);
                    }
                    for (int m = 0; m <= E + F - e - f; ++m) {
                        double r = QC[j] * V(h, gm, m) + WQ[j] * V(h, gm, m + 1);
                        if (gmm >= 0) r += (nf - 1) * oo2e * (V(h, gmm, m) - roe * V(h, gmm, m + 1));
                        if (hm >= 0) r += ne * oo2ze * V(hm, gm, m + 1);
                        V(h, g, m) = r;
                    }
                }
            }
        }
    }
#undef V
}

/* ------------------------------------------------------------------ HRR ------ */
/* Horizontal recurrence on the row index of X.
 * X: rows indexed by global Cartesian index h (>= hoff(la) .. hoff(la+lb+1)), row
 * stride ncol; produces out[(ia*ncart(lb)+ib)*ncol + x] = (a b| for a of AM la and
 * b of AM lb:   (a, b+1_i| = (a+1_i, b| + AB_i (a, b|. */
static void hrr_rows(int la, int lb, const double AB[3], const double *X, int ncol, double *out) {
    if (lb == 0) {
        memcpy(out, X + (size_t)hoff(la) * ncol, sizeof(double) * ncart(la) * ncol);
        return;
    }
    /* level k holds (a, b_k| for a in [la, la+lb-k]; rows (ha - hoff(la)), cols ib */
    int nrow0 = hoff(la + lb + 1) - hoff(la);
    double *prev = (double *)malloc(sizeof(double) * (size_t)nrow0 * ncol);
    memcpy(prev, X + (size_t)hoff(la) * ncol, sizeof(double) * (size_t)nrow0 * ncol);
    int nbprev = 1;
    for (int k = 1; k <= lb; ++k) {
        int nrow = hoff(la + lb - k + 1) - hoff(la);
        int nb = ncart(k);
        double *cur = (double *)malloc(sizeof(double) * (size_t)nrow * nb * ncol);
        for (int ar = 0; ar < nrow; ++ar) {
            int ha = hoff(la) + ar;
            /* recover (lx,ly,lz) of ha */
            int al = 0;
            while (hoff(al + 1) <= ha) ++al;
            const int *xa = g_comp[al][ha - hoff(al)];
            for (int ib = 0; ib < nb; ++ib) {
                const int *xb = g_comp[k][ib];
                int i = xb[0] > 0 ? 0 : (xb[1] > 0 ? 1 : 2);
                int yb[3] = {xb[0], xb[1], xb[2]};
                yb[i] -= 1;
                int ibm = lidx(yb[0], yb[1], yb[2]);
                int ya[3] = {xa[0], xa[1], xa[2]};
                ya[i] += 1;
                int hap = cidx(ya[0], ya[1], ya[2]) - hoff(la);
                double *dst = cur + ((size_t)ar * nb + ib) * ncol;
                const double *s1 = prev + ((size_t)hap * nbprev + ibm) * ncol;
                const double *s2 = prev + ((size_t)ar * nbprev + ibm) * ncol;
                for (int x = 0; x < ncol; ++x) dst[x] = s1[x] + AB[i] * s2[x];
            }
        }
        free(prev);
        prev = cur;
        nbprev = nb;
    }
    memcpy(out, prev, sizeof(double) * (size_t)ncart(la) * ncart(lb) * ncol);
    free(prev);
}

/* X: [NE rows (global e index)][NF cols (global f index)] contracted (e0|f0).
 * Produces (ab|cd) block [na*nb][nc*nd]. */
static void hrr_both(int la, int lb, int lc, int ld, const double AB[3], const double CD[3],
                     const double *X, int NF, double *out) {
    int nab = ncart(la) * ncart(lb);
    double *t1 = (double *)malloc(sizeof(double) * (size_t)nab * NF);
    hrr_rows(la, lb, AB, X, NF, t1);
    /* transpose to [f][ab] */
    double *t2 = (double *)malloc(sizeof(double) * (size_t)nab * NF);
    for (int r = 0; r < nab; ++r)
        for (int f = 0; f < NF; ++f) t2[(size_t)f * nab + r] = t1[(size_t)r * NF + f];
    int ncd = ncart(lc) * ncart(ld);
    double *t3 = (double *)malloc(sizeof(double) * (size_t)ncd * nab);
    hrr_rows(lc, ld, CD, t2, nab, t3);
    for (int r = 0; r < nab; ++r)
        for (int c = 0; c < ncd; ++c) out[(size_t)r * ncd + c] = t3[(size_t)c * nab + r];
    free(t1);
    free(t2);
    free(t3);
}

/* ------------------------------------------------------------- quartets ------ */
typedef struct {
    double *v;
    size_t vcap;
} scratch_t;

static double *scratch_get(scratch_t *s, size_t n) {
    if (n > s->vcap) {
        free(s->v);
        s->v = (double *)malloc(sizeof(double) * n);
        s->vcap = n;
    }
    return s->v;
}

/* Contracted Cartesian shell quartet (s1 s2|s3 s4) into out[n1*n2*n3*n4] row-major.
 * If deriv != 0, out holds 12 blocks (Libint first-derivative buffer order:
 * 3*centre + xyz, centres 0..3 = s1..s4), each n1*n2*n3*n4. */
static int quartet(const qxo_basis *B, int s1, int s2, int s3, int s4, int deriv, double *out,
                   scratch_t *scr) {
    int la = B->l[s1], lb = B->l[s2], lc = B->l[s3], ld = B->l[s4];
    const double *A = B->center + 3 * s1, *Bc = B->center + 3 * s2, *C = B->center + 3 * s3,
                 *D = B->center + 3 * s4;
    double AB[3], CD[3];
    for (int i = 0; i < 3; ++i) { AB[i] = A[i] - Bc[i]; CD[i] = C[i] - D[i]; }
    double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double CD2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    int E = la + lb + (deriv ? 1 : 0), F = lc + ld + (deriv ? 1 : 0);
    int NE = hoff(E + 1), NF = hoff(F + 1), M = E + F + 1;
    size_t vsz = (size_t)NE * NF * M;
    size_t asz = (size_t)NE * NF;
    double *v = scratch_get(scr, vsz + 4 * asz);
    double *U = v + vsz, *WA = U + asz, *WB = WA + asz, *WC = WB + asz;
    memset(U, 0, sizeof(double) * asz * (deriv ? 4 : 1));
    double Fm[4 * QXO_LMAX + 8];
    const double pref0 = 2.0 * pow(M_PI, 2.5);
    for (int p1 = 0; p1 < B->nprim[s1]; ++p1)
        for (int p2 = 0; p2 < B->nprim[s2]; ++p2) {
            double a = B->alpha[B->prim_off[s1] + p1], b = B->alpha[B->prim_off[s2] + p2];
            double ca = B->coef[B->prim_off[s1] + p1], cb = B->coef[B->prim_off[s2] + p2];
            double zeta = a + b;
            double P[3], PA[3];
            /* P - A = -(b / zeta)(A - B): exactly zero for a one-centre pair */
            for (int i = 0; i < 3; ++i) { PA[i] = -(b / zeta) * AB[i]; P[i] = A[i] + PA[i]; }
            double Kab = exp(-a * b / zeta * AB2) * ca * cb;
            for (int p3 = 0; p3 < B->nprim[s3]; ++p3)
                for (int p4 = 0; p4 < B->nprim[s4]; ++p4) {
                    double c = B->alpha[B->prim_off[s3] + p3], d = B->alpha[B->prim_off[s4] + p4];
                    double cc = B->coef[B->prim_off[s3] + p3], cd = B->coef[B->prim_off[s4] + p4];
                    double eta = c + d;
                    double Q[3], QC[3], W[3], WP[3], WQ[3];
                    for (int i = 0; i < 3; ++i) { QC[i] = -(d / eta) * CD[i]; Q[i] = C[i] + QC[i]; }
                    double Kcd = exp(-c * d / eta * CD2) * cc * cd;
                    double rho = zeta * eta / (zeta + eta);
                    double PQ2 = 0.0;
                    for (int i = 0; i < 3; ++i) {
                        /* W - P = -eta/(zeta+eta) (P - Q), P - Q = (A - C) + PA - QC */
                        const double PQ = (A[i] - C[i]) + PA[i] - QC[i];
                        W[i] = P[i] - eta / (zeta + eta) * PQ;
                        WP[i] = -eta / (zeta + eta) * PQ;
                        WQ[i] = zeta / (zeta + eta) * PQ;
                        PQ2 += PQ * PQ;
                    }
                    qxo_boys(E + F, rho * PQ2, Fm);
                    double pref = pref0 / (zeta * eta * sqrt(zeta + eta)) * Kab * Kcd;
                    vrr(E, F, zeta, eta, PA, WP, QC, WQ, rho, Fm, pref, v);
                    const int Mv = M;
                    if (!deriv) {
                        for (size_t h = 0; h < (size_t)NE; ++h)
                            for (int g = 0; g < NF; ++g) U[h * NF + g] += v[(h * NF + g) * Mv];
                    } else {
                        for (size_t h = 0; h < (size_t)NE; ++h)
                            for (int g = 0; g < NF; ++g) {
                                double x = v[(h * NF + g) * Mv];
                                U[h * NF + g] += x;
                                WA[h * NF + g] += 2.0 * a * x;
                                WB[h * NF + g] += 2.0 * b * x;
                                WC[h * NF + g] += 2.0 * c * x;
                            }
                    }
                }
        }
    int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
    size_t nblk = (size_t)na * nb * nc * nd;
    if (!deriv) {
        hrr_both(la, lb, lc, ld, AB, CD, U, NF, out);
        return 0;
    }
    /* shifted blocks */
    double *Ap = (double *)malloc(sizeof(double) * ncart(la + 1) * nb * nc * nd);
    double *Bp = (double *)malloc(sizeof(double) * na * ncart(lb + 1) * nc * nd);
    double *Cp = (double *)malloc(sizeof(double) * na * nb * ncart(lc + 1) * nd);
    double *Am = la ? (double *)malloc(sizeof(double) * ncart(la - 1) * nb * nc * nd) : NULL;
    double *Bm = lb ? (double *)malloc(sizeof(double) * na * ncart(lb - 1) * nc * nd) : NULL;
    double *Cm = lc ? (double *)malloc(sizeof(double) * na * nb * ncart(lc - 1) * nd) : NULL;
    hrr_both(la + 1, lb, lc, ld, AB, CD, WA, NF, Ap);
    hrr_both(la, lb + 1, lc, ld, AB, CD, WB, NF, Bp);
    hrr_both(la, lb, lc + 1, ld, AB, CD, WC, NF, Cp);
    if (la) hrr_both(la - 1, lb, lc, ld, AB, CD, U, NF, Am);
    if (lb) hrr_both(la, lb - 1, lc, ld, AB, CD, U, NF, Bm);
    if (lc) hrr_both(la, lb, lc - 1, ld, AB, CD, U, NF, Cm);
    for (int ia = 0; ia < na; ++ia) {
        const int *xa = g_comp[la][ia];
        for (int ib = 0; ib < nb; ++ib) {
            const int *xb = g_comp[lb][ib];
            for (int ic = 0; ic < nc; ++ic) {
                const int *xc = g_comp[lc][ic];
                for (int id = 0; id < nd; ++id) {
                    size_t o = (((size_t)ia * nb + ib) * nc + ic) * nd + id;
                    for (int i = 0; i < 3; ++i) {
                        int y[3];
                        double dA, dB, dC;
                        /* centre A */
                        y[0] = xa[0]; y[1] = xa[1]; y[2] = xa[2]; y[i] += 1;
                        dA = Ap[(((size_t)lidx(y[0], y[1], y[2]) * nb + ib) * nc + ic) * nd + id];
                        if (xa[i] > 0) {
                            y[i] -= 2;
                            dA -= xa[i] * Am[(((size_t)lidx(y[0], y[1], y[2]) * nb + ib) * nc + ic) * nd + id];
                        }
                        /* centre B */
                        y[0] = xb[0]; y[1] = xb[1]; y[2] = xb[2]; y[i] += 1;
                        dB = Bp[(((size_t)ia * ncart(lb + 1) + lidx(y[0], y[1], y[2])) * nc + ic) * nd + id];
                        if (xb[i] > 0) {
                            y[i] -= 2;
                            dB -= xb[i] * Bm[(((size_t)ia * ncart(lb - 1) + lidx(y[0], y[1], y[2])) * nc + ic) * nd + id];
                        }
                        /* centre C */
                        y[0] = xc[0]; y[1] = xc[1]; y[2] = xc[2]; y[i] += 1;
                        dC = Cp[(((size_t)ia * nb + ib) * ncart(lc + 1) + lidx(y[0], y[1], y[2])) * nd + id];
                        if (xc[i] > 0) {
                            y[i] -= 2;
                            dC -= xc[i] * Cm[(((size_t)ia * nb + ib) * ncart(lc - 1) + lidx(y[0], y[1], y[2])) * nd + id];
                        }
                        out[(0 * 3 + i) * nblk + o] = dA;
                        out[(1 * 3 + i) * nblk + o] = dB;
                        out[(2 * 3 + i) * nblk + o] = dC;
                        out[(3 * 3 + i) * nblk + o] = -(dA + dB + dC);
                    }
                }
            }
        }
    }
    free(Ap); free(Bp); free(Cp); free(Am); free(Bm); free(Cm);
    return 0;
}

static int shell_size(int l) { return ncart(l); }

/* ------------------------------------------------------------- public API ---- */
int qxo_shell_quartet(const qxo_basis *B, int s1, int s2, int s3, int s4, double *out) {
    init_tables();
    scratch_t s = {0, 0};
    int r = quartet(B, s1, s2, s3, s4, 0, out, &s);
    free(s.v);
    return r;
}

int qxo_shell_quartet_deriv1(const qxo_basis *B, int s1, int s2, int s3, int s4, double *out) {
    init_tables();
    scratch_t s = {0, 0};
    int r = quartet(B, s1, s2, s3, s4, 1, out, &s);
    free(s.v);
    return r;
}

static int nthreads_of(int req) {
#ifdef _OPENMP
    return req > 0 ? req : omp_get_max_threads();
#else
    (void)req;
    return 1;
#endif
}

/* Schwarz table (libint_interface.cc:158-229): K[s1*ns+s2] = max |(f1 f2|f1 f2)|,
 * symmetric; returns max K in *kmax. */
int qxo_schwarz(const qxo_basis *B, double *K, double *kmax, int nthreads) {
    init_tables();
    int ns = B->nshell;
    double mx = 0.0;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt) reduction(max : mx)
    {
        scratch_t scr = {0, 0};
        double *buf = NULL;
        size_t cap = 0;
#pragma omp for schedule(dynamic)
        for (int s1 = 0; s1 < ns; ++s1)
            for (int s2 = 0; s2 <= s1; ++s2) {
                int n1 = shell_size(B->l[s1]), n2 = shell_size(B->l[s2]);
                size_t need = (size_t)n1 * n2 * n1 * n2;
                if (need > cap) { free(buf); buf = (double *)malloc(sizeof(double) * need); cap = need; }
                quartet(B, s1, s2, s1, s2, 0, buf, &scr);
                double v = 0.0;
                for (int f1 = 0; f1 < n1; ++f1)
                    for (int f2 = 0; f2 < n2; ++f2) {
                        double x = fabs(buf[f1 * (n1 * n2 * n2 + n2) + f2 * (n1 * n2 + 1)]);
                        if (x > v) v = x;
                    }
                K[s1 * ns + s2] = K[s2 * ns + s1] = v;
                if (v > mx) mx = v;
            }
        free(buf);
        free(scr.v);
    }
    *kmax = mx;
    return 0;
}

/* Screened pair list (s1 >= s2), reference order; returns count. pairs[2*k]=s1. */
int qxo_pairs(const qxo_basis *B, const double *K, double kmax, double thr, int *pairs) {
    int ns = B->nshell, n = 0;
    double cut = thr * thr / kmax;
    for (int s1 = 0; s1 < ns; ++s1)
        for (int s2 = 0; s2 <= s1; ++s2)
            if (K[s1 * ns + s2] >= cut) {
                pairs[2 * n] = s1;
                pairs[2 * n + 1] = s2;
                ++n;
            }
    return n;
}

static void shell2bf_of(const qxo_basis *B, long *s2bf, long *nbf) {
    long o = 0;
    for (int s = 0; s < B->nshell; ++s) { s2bf[s] = o; o += shell_size(B->l[s]); }
    *nbf = o;
}

/* Dense ERI tensor with the reference's loops and scatter (libint_interface.cc:486-647). */
int qxo_compute_2e_int(const qxo_basis *B, double thr, double *out, int nthreads) {
    init_tables();
    int ns = B->nshell;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    memset(out, 0, sizeof(double) * (size_t)n * n * n * n);
    double thr2 = thr * thr;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt)
    {
        scratch_t scr = {0, 0};
        double *buf = (double *)malloc(sizeof(double) * 50625 * 16);
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            for (int jp = 0; jp < np; ++jp) {
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                quartet(B, p1, p2, p3, p4, 0, buf, &scr);
                int n1 = shell_size(B->l[p1]), n2 = shell_size(B->l[p2]), n3 = shell_size(B->l[p3]),
                    n4 = shell_size(B->l[p4]);
                long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
                for (int f1 = 0, idx = 0; f1 < n1; ++f1)
                    for (int f2 = 0; f2 < n2; ++f2)
                        for (int f3 = 0; f3 < n3; ++f3)
                            for (int f4 = 0; f4 < n4; ++f4, ++idx) {
                                long i = b1 + f1, j = b2 + f2, k = b3 + f3, l = b4 + f4;
                                double x = buf[idx];
                                out[((i * n + j) * n + k) * n + l] = x;
                                if (p1 != p2) out[((j * n + i) * n + k) * n + l] = x;
                                if (p3 != p4) out[((i * n + j) * n + l) * n + k] = x;
                                if (p1 != p2 && p3 != p4) out[((j * n + i) * n + l) * n + k] = x;
                            }
            }
        }
        free(buf);
        free(scr.v);
    }
    free(K); free(pairs); free(s2bf);
    return 0;
}

/* First-derivative tensor (3N, n,n,n,n) with the reference's semantics
 * (libint_interface.cc:2582-2779).  If deriv_idx >= 0 only that nuclear slice is
 * produced (compute_2e_deriv with a one-hot deriv_vec, libint_interface.cc:1097-1335),
 * into out[n^4]. */
int qxo_eri_deriv1(const qxo_basis *B, double thr, int deriv_idx, double *out, int nthreads) {
    init_tables();
    int ns = B->nshell;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    size_t n4 = (size_t)n * n * n * n;
    int nslice = deriv_idx >= 0 ? 1 : 3 * B->natom;
    memset(out, 0, sizeof(double) * n4 * nslice);
    double thr2 = thr * thr;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt)
    {
        scratch_t scr = {0, 0};
        double *buf = (double *)malloc(sizeof(double) * 50625 * 12);
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            for (int jp = 0; jp < np; ++jp) {
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                int at[4] = {B->atom[p1], B->atom[p2], B->atom[p3], B->atom[p4]};
                if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
                if (deriv_idx >= 0) {
                    int da = deriv_idx / 3;
                    if (at[0] != da && at[1] != da && at[2] != da && at[3] != da) continue;
                }
                quartet(B, p1, p2, p3, p4, 1, buf, &scr);
                int n1 = shell_size(B->l[p1]), n2 = shell_size(B->l[p2]), n3 = shell_size(B->l[p3]),
                    nn4 = shell_size(B->l[p4]);
                size_t nblk = (size_t)n1 * n2 * n3 * nn4;
                long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
                for (int s = 0; s < nslice; ++s) {
                    int nuc = deriv_idx >= 0 ? deriv_idx : s;
                    int atom = nuc / 3, xyz = nuc % 3;
                    int use[4], nuse = 0;
                    for (int c = 0; c < 4; ++c)
                        if (at[c] == atom) use[nuse++] = 3 * c + xyz;
                    if (!nuse) continue;
                    double *o = out + (size_t)s * n4;
                    for (int f1 = 0, idx = 0; f1 < n1; ++f1)
                        for (int f2 = 0; f2 < n2; ++f2)
                            for (int f3 = 0; f3 < n3; ++f3)
                                for (int f4 = 0; f4 < nn4; ++f4, ++idx) {
                                    double x = 0.0;
                                    for (int u = 0; u < nuse; ++u) x += buf[use[u] * nblk + idx];
                                    long i = b1 + f1, j = b2 + f2, k = b3 + f3, l = b4 + f4;
                                    o[((i * n + j) * n + k) * n + l] += x;
                                    if (p1 != p2) o[((j * n + i) * n + k) * n + l] += x;
                                    if (p3 != p4) o[((i * n + j) * n + l) * n + k] += x;
                                    if (p1 != p2 && p3 != p4) o[((j * n + i) * n + l) * n + k] += x;
                                }
                }
            }
        }
        free(buf);
        free(scr.v);
    }
    free(K); free(pairs); free(s2bf);
    return 0;
}

/* Contracted gradient  g[3N] = sum_ijkl Gamma_ijkl d(ij|kl)/dR  with
 * Gamma_ijkl = cj * D_ij D_kl + ck * D_ik D_jl  (HF: cj = 1, ck = -1/2),
 * evaluated over 8-fold-unique screened quartets with degeneracy weights.
 * Quartet screening as the reference's (pair list + K_ab K_cd >= thr^2).
 * This is the oracle for the adjoint gradient. */
int qxo_grad_contract(const qxo_basis *B, double thr, const double *Dm, double cj, double ck,
                      double *grad, int nthreads) {
    init_tables();
    int ns = B->nshell;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    int N3 = 3 * B->natom;
    memset(grad, 0, sizeof(double) * N3);
    double thr2 = thr * thr;
    int nt = nthreads_of(nthreads);
#define GAM(i, j, k, l) (cj * Dm[(i) * n + (j)] * Dm[(k) * n + (l)] + ck * Dm[(i) * n + (k)] * Dm[(j) * n + (l)])
#pragma omp parallel num_threads(nt)
    {
        scratch_t scr = {0, 0};
        double *buf = (double *)malloc(sizeof(double) * 50625 * 12);
        double *g = (double *)calloc(N3, sizeof(double));
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            for (int jp = 0; jp <= ip; ++jp) {
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                int at[4] = {B->atom[p1], B->atom[p2], B->atom[p3], B->atom[p4]};
                if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
                quartet(B, p1, p2, p3, p4, 1, buf, &scr);
                int n1 = shell_size(B->l[p1]), n2 = shell_size(B->l[p2]), n3 = shell_size(B->l[p3]),
                    nn4 = shell_size(B->l[p4]);
                size_t nblk = (size_t)n1 * n2 * n3 * nn4;
                long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
                double acc[12] = {0};
                for (int f1 = 0, idx = 0; f1 < n1; ++f1)
                    for (int f2 = 0; f2 < n2; ++f2)
                        for (int f3 = 0; f3 < n3; ++f3)
                            for (int f4 = 0; f4 < nn4; ++f4, ++idx) {
                                long i = b1 + f1, j = b2 + f2, k = b3 + f3, l = b4 + f4;
                                double w = GAM(i, j, k, l);
                                if (p1 != p2) w += GAM(j, i, k, l);
                                if (p3 != p4) w += GAM(i, j, l, k);
                                if (p1 != p2 && p3 != p4) w += GAM(j, i, l, k);
                                if (ip != jp) {
                                    w += GAM(k, l, i, j);
                                    if (p3 != p4) w += GAM(l, k, i, j);
                                    if (p1 != p2) w += GAM(k, l, j, i);
                                    if (p1 != p2 && p3 != p4) w += GAM(l, k, j, i);
                                }
                                for (int c = 0; c < 12; ++c) acc[c] += w * buf[c * nblk + idx];
                            }
                for (int c = 0; c < 4; ++c)
                    for (int x = 0; x < 3; ++x) g[3 * at[c] + x] += acc[3 * c + x];
            }
        }
#pragma omp critical
        for (int i = 0; i < N3; ++i) grad[i] += g[i];
        free(g);
        free(buf);
        free(scr.v);
    }
#undef GAM
    free(K); free(pairs); free(s2bf);
    return 0;
}

/* Contracted blocks of a list of shell quartets (q4[4*q + 0..3], in the given
 * centre order), all of one angular-momentum class: out[q * nblk + element],
 * element row-major over (f1, f2, f3, f4).  For comparing a unique layout
 * quartet by quartet. */
int qxo_quartet_blocks(const qxo_basis *B, const int *q4, long nq, double *out, int nthreads) {
    init_tables();
    if (nq <= 0) return 0;
    const int *q0 = q4;
    size_t nblk = (size_t)ncart(B->l[q0[0]]) * ncart(B->l[q0[1]]) * ncart(B->l[q0[2]]) * ncart(B->l[q0[3]]);
    for (long q = 0; q < nq; ++q)
        for (int c = 0; c < 4; ++c)
            if (B->l[q4[4 * q + c]] != B->l[q0[c]]) return -1;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt)
    {
        scratch_t scr = {0, 0};
#pragma omp for schedule(dynamic, 64)
        for (long q = 0; q < nq; ++q)
            quartet(B, q4[4 * q], q4[4 * q + 1], q4[4 * q + 2], q4[4 * q + 3], 0, out + (size_t)q * nblk, &scr);
        free(scr.v);
    }
    return 0;
}

/* Adjoint-gradient contribution of a list of 8-fold-unique shell quartets
 * (q4[4*q + 0..3]): grad[3*atom + xyz] += sum over the quartets' distinct images
 * of Gamma_ijkl d(ij|kl)/dR, Gamma = cj D_ij D_kl + ck D_ik D_jl -- the terms
 * qxo_grad_contract adds for the same quartets.  grad is not zeroed. */
int qxo_grad_quartets(const qxo_basis *B, const int *q4, long nq, const double *Dm, double cj, double ck,
                      double *grad, int nthreads) {
    init_tables();
    int ns = B->nshell;
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    int N3 = 3 * B->natom;
    int nt = nthreads_of(nthreads);
#define GAM(i, j, k, l) (cj * Dm[(i) * n + (j)] * Dm[(k) * n + (l)] + ck * Dm[(i) * n + (k)] * Dm[(j) * n + (l)])
#pragma omp parallel num_threads(nt)
    {
        scratch_t scr = {0, 0};
        double *buf = (double *)malloc(sizeof(double) * 10000 * 12);
        double *g = (double *)calloc(N3, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (long q = 0; q < nq; ++q) {
            int p1 = q4[4 * q], p2 = q4[4 * q + 1], p3 = q4[4 * q + 2], p4 = q4[4 * q + 3];
            int at[4] = {B->atom[p1], B->atom[p2], B->atom[p3], B->atom[p4]};
            if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
            int sPQ = !((p1 == p3 && p2 == p4) || (p1 == p4 && p2 == p3));
            quartet(B, p1, p2, p3, p4, 1, buf, &scr);
            int n1 = shell_size(B->l[p1]), n2 = shell_size(B->l[p2]), n3 = shell_size(B->l[p3]),
                nn4 = shell_size(B->l[p4]);
            size_t nblk = (size_t)n1 * n2 * n3 * nn4;
            long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
            double acc[12] = {0};
            for (int f1 = 0, idx = 0; f1 < n1; ++f1)
                for (int f2 = 0; f2 < n2; ++f2)
                    for (int f3 = 0; f3 < n3; ++f3)
                        for (int f4 = 0; f4 < nn4; ++f4, ++idx) {
                            long i = b1 + f1, j = b2 + f2, k = b3 + f3, l = b4 + f4;
                            double w = GAM(i, j, k, l);
                            if (p1 != p2) w += GAM(j, i, k, l);
                            if (p3 != p4) w += GAM(i, j, l, k);
                            if (p1 != p2 && p3 != p4) w += GAM(j, i, l, k);
                            if (sPQ) {
                                w += GAM(k, l, i, j);
                                if (p3 != p4) w += GAM(l, k, i, j);
                                if (p1 != p2) w += GAM(k, l, j, i);
                                if (p1 != p2 && p3 != p4) w += GAM(l, k, j, i);
                            }
                            for (int c = 0; c < 12; ++c) acc[c] += w * buf[c * nblk + idx];
                        }
            for (int c = 0; c < 4; ++c)
                for (int x = 0; x < 3; ++x) g[3 * at[c] + x] += acc[3 * c + x];
        }
#pragma omp critical
        for (int i = 0; i < N3; ++i) grad[i] += g[i];
        free(g);
        free(buf);
        free(scr.v);
    }
#undef GAM
    free(s2bf);
    return 0;
}

/* Time-bounded unique-quartet evaluation for the CPU baseline: evaluates the
 * screened 8-fold-unique quartets whose linear index (in bra-major, ket <= bra
 * order over the reference pair list) is congruent to `phase` modulo `stride`,
 * discarding results; returns the number of quartets evaluated.  K_in (the Schwarz
 * table of qxo_schwarz) may be passed so the call times quartet work only.  deriv selects
 * the first-derivative engine.  checksum receives a sum of the first element of
 * every block so the work cannot be optimised away. */
long qxo_unique_sample(const qxo_basis *B, double thr, long stride, long phase, int deriv, const double *K_in,
                       double kmax_in, double *checksum, int nthreads) {
    init_tables();
    int ns = B->nshell;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    if (K_in) {
        memcpy(K, K_in, sizeof(double) * ns * ns);
        kmax = kmax_in;
    } else {
        qxo_schwarz(B, K, &kmax, nthreads);
    }
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    double thr2 = thr * thr;
    long count = 0;
    double cs = 0.0;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt) reduction(+ : count, cs)
    {
        scratch_t scr = {0, 0};
        double *buf = (double *)malloc(sizeof(double) * 50625 * 12);
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            long base = (long)ip * (ip + 1) / 2;
            for (int jp = 0; jp <= ip; ++jp) {
                if ((base + jp) % stride != phase) continue;
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                quartet(B, p1, p2, p3, p4, deriv, buf, &scr);
                cs += buf[0];
                ++count;
            }
        }
        free(buf);
        free(scr.v);
    }
    *checksum = cs;
    free(K); free(pairs);
    return count;
}

/* Count of screened 8-fold-unique quartets (the throughput unit). */
long qxo_count_unique(const qxo_basis *B, double thr, int nthreads) {
    int ns = B->nshell;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    init_tables();
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    double thr2 = thr * thr;
    long c = 0;
    for (int ip = 0; ip < np; ++ip)
        for (int jp = 0; jp <= ip; ++jp)
            if (K[pairs[2 * ip] * ns + pairs[2 * ip + 1]] * K[pairs[2 * jp] * ns + pairs[2 * jp + 1]] >= thr2) ++c;
    free(K); free(pairs);
    return c;
}


/* (a b|c d) block of a weighted set for AMs shifted by (da, db, dc) (d unchanged),
 * cached in *slot. */
static double *blk2(const qxo_basis *B, const int *L, const double *AB, const double *CD, const double *X, int NF,
                    double *cached, double **slot, int da, int db, int dc) {
    (void)B;
    if (cached) return cached;
    int la = L[0] + da, lb = L[1] + db, lc = L[2] + dc, ld = L[3];
    size_t sz = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    double *o = (double *)malloc(sizeof(double) * sz);
    hrr_both(la, lb, lc, ld, AB, CD, X, NF, o);
    *slot = o;
    return o;
}

/* ------------------------------------------------------- second derivatives --- */
/* ------------------------------------------------------- second derivatives --- */
/* Full 12 x 12 block set of second derivatives of the Cartesian quartet block
 * (s1 s2|s3 s4): out[(P*12 + Q) * nblk + o], P, Q = 3*centre + xyz.  Applies
 * d/dA_i g_a = 2 alpha g_{a+1_i} - a_i g_{a-1_i} twice (same-centre and cross-centre
 * terms from ten weighted primitive sums), and the D-centre rows by translational
 * invariance. */
static int quartet2(const qxo_basis *B, int s1, int s2, int s3, int s4, double *out) {
    int L[4] = {B->l[s1], B->l[s2], B->l[s3], B->l[s4]};
    int sh[4] = {s1, s2, s3, s4};
    const double *Cn[4];
    for (int c = 0; c < 4; ++c) Cn[c] = B->center + 3 * sh[c];
    double AB[3], CD[3];
    for (int i = 0; i < 3; ++i) { AB[i] = Cn[0][i] - Cn[1][i]; CD[i] = Cn[2][i] - Cn[3][i]; }
    double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double CD2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    int E = L[0] + L[1] + 2, F = L[2] + L[3] + 2;
    int NE = hoff(E + 1), NF = hoff(F + 1), M = E + F + 1;
    size_t vsz = (size_t)NE * NF * M, asz = (size_t)NE * NF;
    /* sets: 0 U, 1 A, 2 B, 3 C, 4 AA, 5 BB, 6 CC, 7 AB, 8 AC, 9 BC */
    double *v = (double *)malloc(sizeof(double) * (vsz + 10 * asz));
    double *S = v + vsz;
    memset(S, 0, sizeof(double) * 10 * asz);
    double Fm[4 * QXO_LMAX + 8];
    const double pref0 = 2.0 * pow(M_PI, 2.5);
    for (int p1 = 0; p1 < B->nprim[s1]; ++p1)
        for (int p2 = 0; p2 < B->nprim[s2]; ++p2) {
            double a = B->alpha[B->prim_off[s1] + p1], b = B->alpha[B->prim_off[s2] + p2];
            double zeta = a + b, P[3], PA[3];
            for (int i = 0; i < 3; ++i) { PA[i] = -(b / zeta) * AB[i]; P[i] = Cn[0][i] + PA[i]; }
            double Kab = exp(-a * b / zeta * AB2) * B->coef[B->prim_off[s1] + p1] * B->coef[B->prim_off[s2] + p2];
            for (int p3 = 0; p3 < B->nprim[s3]; ++p3)
                for (int p4 = 0; p4 < B->nprim[s4]; ++p4) {
                    double c = B->alpha[B->prim_off[s3] + p3], d = B->alpha[B->prim_off[s4] + p4];
                    double eta = c + d, Q[3], QC[3], W[3], WP[3], WQ[3], PQ2 = 0.0;
                    for (int i = 0; i < 3; ++i) { QC[i] = -(d / eta) * CD[i]; Q[i] = Cn[2][i] + QC[i]; }
                    double Kcd = exp(-c * d / eta * CD2) * B->coef[B->prim_off[s3] + p3] * B->coef[B->prim_off[s4] + p4];
                    double rho = zeta * eta / (zeta + eta);
                    for (int i = 0; i < 3; ++i) {
                        const double PQ = (Cn[0][i] - Cn[2][i]) + PA[i] - QC[i];
                        W[i] = P[i] - eta / (zeta + eta) * PQ;
                        WP[i] = -eta / (zeta + eta) * PQ;
                        WQ[i] = zeta / (zeta + eta) * PQ;
                        PQ2 += PQ * PQ;
                    }
                    qxo_boys(E + F, rho * PQ2, Fm);
                    vrr(E, F, zeta, eta, PA, WP, QC, WQ, rho, Fm, pref0 / (zeta * eta * sqrt(zeta + eta)) * Kab * Kcd, v);
                    double w2[10] = {1.0, 2 * a, 2 * b, 2 * c, 4 * a * a, 4 * b * b, 4 * c * c, 4 * a * b, 4 * a * c, 4 * b * c};
                    for (size_t h = 0; h < (size_t)NE; ++h)
                        for (int g = 0; g < NF; ++g) {
                            double x = v[(h * NF + g) * M];
                            for (int k = 0; k < 10; ++k) S[k * asz + h * NF + g] += w2[k] * x;
                        }
                }
        }
    int n[4];
    for (int c = 0; c < 4; ++c) n[c] = ncart(L[c]);
    size_t nblk = (size_t)n[0] * n[1] * n[2] * n[3];
    /* shifted blocks: cache by (set, dla, dlb, dlc) with shifts in {-2..2} */
    double *cache[10][5][5][5];
    memset(cache, 0, sizeof cache);
#define BLK(set, da, db, dc) blk2(B, L, AB, CD, S + (set) * asz, NF, cache[set][(da) + 2][(db) + 2][(dc) + 2], &cache[set][(da) + 2][(db) + 2][(dc) + 2], da, db, dc)
    for (int P1 = 0; P1 < 9; ++P1)
        for (int Q1 = 0; Q1 < 9; ++Q1) {
            int X = P1 / 3, i = P1 % 3, Y = Q1 / 3, j = Q1 % 3;
            double *dst = out + ((size_t)P1 * 12 + Q1) * nblk;
            for (int ia = 0; ia < n[0]; ++ia)
                for (int ib = 0; ib < n[1]; ++ib)
                    for (int ic = 0; ic < n[2]; ++ic)
                        for (int id = 0; id < n[3]; ++id) {
                            const int *xs[4] = {g_comp[L[0]][ia], g_comp[L[1]][ib], g_comp[L[2]][ic], g_comp[L[3]][id]};
                            int comp[4][3];
                            for (int cc = 0; cc < 4; ++cc)
                                for (int k = 0; k < 3; ++k) comp[cc][k] = xs[cc][k];
                            double val = 0.0;
                            /* enumerate the two derivative factors: each is (+1, weight set, shift +1)
                             * or (-n, unweighted, shift -1) on its centre */
                            for (int fx = 0; fx < 2; ++fx)
                                for (int fy = 0; fy < 2; ++fy) {
                                    int cm[4][3];
                                    memcpy(cm, comp, sizeof cm);
                                    double coef = 1.0;
                                    if (fx == 0) cm[X][i] += 1;
                                    else { coef *= -cm[X][i]; cm[X][i] -= 1; }
                                    if (coef == 0.0) continue;
                                    if (fy == 0) cm[Y][j] += 1;
                                    else { coef *= -cm[Y][j]; cm[Y][j] -= 1; }
                                    if (coef == 0.0) continue;
                                    int neg = 0;
                                    for (int cc = 0; cc < 4; ++cc)
                                        for (int k = 0; k < 3; ++k)
                                            if (cm[cc][k] < 0) neg = 1;
                                    if (neg) continue;
                                    /* weight set: product of the factors' weights */
                                    int wX = fx == 0 ? X + 1 : 0, wY = fy == 0 ? Y + 1 : 0; /* 1 A, 2 B, 3 C */
                                    int set;
                                    if (!wX && !wY) set = 0;
                                    else if (!wX || !wY) set = wX ? wX : wY;
                                    else {
                                        int u = wX < wY ? wX : wY, w = wX < wY ? wY : wX;
                                        set = (u == w) ? 3 + u : (u == 1 ? (w == 2 ? 7 : 8) : 9);
                                    }
                                    int dl[4];
                                    for (int cc = 0; cc < 4; ++cc) dl[cc] = cm[cc][0] + cm[cc][1] + cm[cc][2] - L[cc];
                                    double *bk = BLK(set, dl[0], dl[1], dl[2]);
                                    int nb2 = ncart(L[1] + dl[1]), nc2 = ncart(L[2] + dl[2]);
                                    size_t o = (((size_t)lidx(cm[0][0], cm[0][1], cm[0][2]) * nb2 + lidx(cm[1][0], cm[1][1], cm[1][2])) * nc2 +
                                                lidx(cm[2][0], cm[2][1], cm[2][2])) * n[3] + lidx(cm[3][0], cm[3][1], cm[3][2]);
                                    val += coef * bk[o];
                                }
                            dst[(((size_t)ia * n[1] + ib) * n[2] + ic) * n[3] + id] = val;
                        }
        }
    /* D rows and columns by translational invariance */
    for (int i = 0; i < 3; ++i)
        for (int Q1 = 0; Q1 < 9; ++Q1) {
            double *dD = out + ((size_t)(9 + i) * 12 + Q1) * nblk, *dT = out + ((size_t)Q1 * 12 + 9 + i) * nblk;
            for (size_t o = 0; o < nblk; ++o) {
                double s = 0.0;
                for (int X = 0; X < 3; ++X) s += out[((size_t)(3 * X + i) * 12 + Q1) * nblk + o];
                dD[o] = -s;
                dT[o] = -s;
            }
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double *dst = out + ((size_t)(9 + i) * 12 + 9 + j) * nblk;
            for (size_t o = 0; o < nblk; ++o) {
                double s = 0.0;
                for (int X = 0; X < 3; ++X) s += out[((size_t)(9 + i) * 12 + 3 * X + j) * nblk + o];
                dst[o] = -s;
            }
        }
#undef BLK
    for (int a = 0; a < 10; ++a)
        for (int b = 0; b < 5; ++b)
            for (int c = 0; c < 5; ++c)
                for (int d = 0; d < 5; ++d) free(cache[a][b][c][d]);
    free(v);
    return 0;
}

int qxo_shell_quartet_deriv2(const qxo_basis *B, int s1, int s2, int s3, int s4, double *out) {
    init_tables();
    return quartet2(B, s1, s2, s3, s4, out);
}

/* Second-derivative tensor with the reference's semantics
 * (libint_interface.cc:2582-2779 at deriv_order 2; compute_2e_deriv :1097-1335):
 * unique nuclear pairs nu1 <= nu2 in the order of generate_multi_index_lookup(3N, 2);
 * element = sum over shell positions p on atom(nu1), q on atom(nu2) of the
 * Libint buffer for the sorted pair (3p + c1, 3q + c2).  If pair_idx >= 0 only
 * that slice is produced. */
int qxo_eri_deriv2(const qxo_basis *B, double thr, int pair_idx, double *out, int nthreads) {
    init_tables();
    int ns = B->nshell, N3 = 3 * B->natom;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    size_t n4 = (size_t)n * n * n * n;
    int npair = N3 * (N3 + 1) / 2;
    int nslice = pair_idx >= 0 ? 1 : npair;
    memset(out, 0, sizeof(double) * n4 * nslice);
    int *nu1 = (int *)malloc(sizeof(int) * npair), *nu2 = (int *)malloc(sizeof(int) * npair);
    for (int a = 0, k = 0; a < N3; ++a)
        for (int b = a; b < N3; ++b, ++k) { nu1[k] = a; nu2[k] = b; }
    double thr2 = thr * thr;
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt)
    {
        int lmx = 0;
        for (int s = 0; s < ns; ++s) lmx = B->l[s] > lmx ? B->l[s] : lmx;
        size_t nb = (size_t)ncart(lmx) * ncart(lmx) * ncart(lmx) * ncart(lmx);
        double *buf = (double *)malloc(sizeof(double) * nb * 144);
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            for (int jp = 0; jp < np; ++jp) {
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                int at[4] = {B->atom[p1], B->atom[p2], B->atom[p3], B->atom[p4]};
                if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
                quartet2(B, p1, p2, p3, p4, buf);
                int nn[4] = {shell_size(B->l[p1]), shell_size(B->l[p2]), shell_size(B->l[p3]), shell_size(B->l[p4])};
                size_t nblk = (size_t)nn[0] * nn[1] * nn[2] * nn[3];
                long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
                for (int s = 0; s < nslice; ++s) {
                    int k = pair_idx >= 0 ? pair_idx : s;
                    int A1 = nu1[k] / 3, c1 = nu1[k] % 3, A2 = nu2[k] / 3, c2 = nu2[k] % 3;
                    int P[4], Q[4], nP = 0, nQ = 0;
                    for (int c = 0; c < 4; ++c) {
                        if (at[c] == A1) P[nP++] = 3 * c + c1;
                        if (at[c] == A2) Q[nQ++] = 3 * c + c2;
                    }
                    if (!nP || !nQ) continue;
                    double *o = out + (size_t)s * n4;
                    for (int f1 = 0, idx = 0; f1 < nn[0]; ++f1)
                        for (int f2 = 0; f2 < nn[1]; ++f2)
                            for (int f3 = 0; f3 < nn[2]; ++f3)
                                for (int f4 = 0; f4 < nn[3]; ++f4, ++idx) {
                                    double x = 0.0;
                                    for (int u = 0; u < nP; ++u)
                                        for (int w = 0; w < nQ; ++w) {
                                            int lo = P[u] < Q[w] ? P[u] : Q[w], hi = P[u] < Q[w] ? Q[w] : P[u];
                                            x += buf[((size_t)lo * 12 + hi) * nblk + idx];
                                        }
                                    long i = b1 + f1, j = b2 + f2, kk = b3 + f3, l = b4 + f4;
                                    o[((i * n + j) * n + kk) * n + l] += x;
                                    if (p1 != p2) o[((j * n + i) * n + kk) * n + l] += x;
                                    if (p3 != p4) o[((i * n + j) * n + l) * n + kk] += x;
                                    if (p1 != p2 && p3 != p4) o[((j * n + i) * n + l) * n + kk] += x;
                                }
                }
            }
        }
        free(buf);
    }
    free(K); free(pairs); free(s2bf); free(nu1); free(nu2);
    return 0;
}

/* ------------------------------------------------------ derivatives of order k --- */
int qxo_multi_index_lookup(int nparams, int order, int *out);
/* Rank of (e0, e1, e2, e3) >= 0 with sum <= K among such tuples, lexicographic. */
static long binom_l(int n, int k) {
    if (k < 0 || k > n) return 0;
    long r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}
static int set_rank(int K, const int *e) {
    int r = 0;
    for (int v = 0; v < e[0]; ++v) r += (int)binom_l(K - v + 3, 3);
    for (int v = 0; v < e[1]; ++v) r += (int)binom_l(K - e[0] - v + 2, 2);
    for (int v = 0; v < e[2]; ++v) r += (int)binom_l(K - e[0] - e[1] - v + 1, 1);
    return r + e[3];
}

/* Coefficients of (d/dX)^n on a 1-D Gaussian index i with unit exponent weight:
 * d g_i = [2 alpha] g_{i+1} - i g_{i-1}; cf[j] multiplies (2 alpha)^j g_{i+2j-n}. */
static void dexp1(int n, int i, double *cf) {
    double c[9] = {1, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int s = 0; s < n; ++s) {
        double nc[9] = {0};
        for (int j = 0; j <= s; ++j) {
            int sh = 2 * j - s;
            nc[j + 1] += c[j];
            nc[j] -= (double)(i + sh) * c[j];
        }
        memcpy(c, nc, sizeof c);
    }
    memcpy(cf, c, sizeof(double) * (n + 1));
}

/* All derivative blocks of order k (1..4) of the Cartesian quartet (s1 s2|s3 s4),
 * every centre differentiated directly (no translational invariance):
 * out[m * nblk + o], m = rank of the sorted k-tuple of centre-directions
 * (3 * centre + xyz) among all such tuples over 12 values (Libint's order of
 * derivative buffers), o = block element.  Obara-Saika VRR of [e0|f0] raised by k
 * on each side, accumulated over primitives in weighted sets
 * (2a)^eA (2b)^eB (2c)^eC (2d)^eD, sum e <= k; the derivative identity applied
 * per centre and direction picks the set and the shifted block (HRR cached). */
static int quartetk(const qxo_basis *B, int s1, int s2, int s3, int s4, int k, double *out) {
    if (k < 1 || k > 4) return -1;
    int L[4] = {B->l[s1], B->l[s2], B->l[s3], B->l[s4]};
    int sh[4] = {s1, s2, s3, s4};
    const double *Cn[4];
    for (int c = 0; c < 4; ++c) Cn[c] = B->center + 3 * sh[c];
    double AB[3], CD[3];
    for (int i = 0; i < 3; ++i) { AB[i] = Cn[0][i] - Cn[1][i]; CD[i] = Cn[2][i] - Cn[3][i]; }
    double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    double CD2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    int E = L[0] + L[1] + k, F = L[2] + L[3] + k;
    int NE = hoff(E + 1), NF = hoff(F + 1), M = E + F + 1;
    size_t vsz = (size_t)NE * NF * M, asz = (size_t)NE * NF;
    int NS = (int)binom_l(k + 4, 4);
    double *v = (double *)malloc(sizeof(double) * (vsz + NS * asz));
    double *S = v + vsz;
    memset(S, 0, sizeof(double) * NS * asz);
    int sets[70][4], ns = 0;
    for (int a = 0; a <= k; ++a)
        for (int b = 0; a + b <= k; ++b)
            for (int c = 0; a + b + c <= k; ++c)
                for (int d = 0; a + b + c + d <= k; ++d) {
                    sets[ns][0] = a; sets[ns][1] = b; sets[ns][2] = c; sets[ns][3] = d;
                    ++ns;
                }
    double Fm[4 * QXO_LMAX + 8];
    const double pref0 = 2.0 * pow(M_PI, 2.5);
    for (int p1 = 0; p1 < B->nprim[s1]; ++p1)
        for (int p2 = 0; p2 < B->nprim[s2]; ++p2) {
            double a = B->alpha[B->prim_off[s1] + p1], b = B->alpha[B->prim_off[s2] + p2];
            double zeta = a + b, P[3], PA[3];
            for (int i = 0; i < 3; ++i) { PA[i] = -(b / zeta) * AB[i]; P[i] = Cn[0][i] + PA[i]; }
            double Kab = exp(-a * b / zeta * AB2) * B->coef[B->prim_off[s1] + p1] * B->coef[B->prim_off[s2] + p2];
            for (int p3 = 0; p3 < B->nprim[s3]; ++p3)
                for (int p4 = 0; p4 < B->nprim[s4]; ++p4) {
                    double c = B->alpha[B->prim_off[s3] + p3], d = B->alpha[B->prim_off[s4] + p4];
                    double eta = c + d, Q[3], QC[3], WP[3], WQ[3], PQ2 = 0.0;
                    for (int i = 0; i < 3; ++i) { QC[i] = -(d / eta) * CD[i]; Q[i] = Cn[2][i] + QC[i]; }
                    double Kcd = exp(-c * d / eta * CD2) * B->coef[B->prim_off[s3] + p3] * B->coef[B->prim_off[s4] + p4];
                    double rho = zeta * eta / (zeta + eta);
                    for (int i = 0; i < 3; ++i) {
                        double PQ = (Cn[0][i] - Cn[2][i]) + PA[i] - QC[i];
                        WP[i] = -eta / (zeta + eta) * PQ;
                        WQ[i] = zeta / (zeta + eta) * PQ;
                        PQ2 += PQ * PQ;
                    }
                    (void)P; (void)Q;
                    qxo_boys(E + F, rho * PQ2, Fm);
                    vrr(E, F, zeta, eta, PA, WP, QC, WQ, rho, Fm, pref0 / (zeta * eta * sqrt(zeta + eta)) * Kab * Kcd, v);
                    double e2[4] = {2 * a, 2 * b, 2 * c, 2 * d};
                    for (int q = 0; q < ns; ++q) {
                        double w = 1.0;
                        for (int cc = 0; cc < 4; ++cc)
                            for (int t = 0; t < sets[q][cc]; ++t) w *= e2[cc];
                        double *Sq = S + (size_t)set_rank(k, sets[q]) * asz;
                        for (size_t h = 0; h < (size_t)NE; ++h)
                            for (int g = 0; g < NF; ++g) Sq[h * NF + g] += w * v[(h * NF + g) * M];
                    }
                }
        }
    int n[4];
    for (int c = 0; c < 4; ++c) n[c] = ncart(L[c]);
    size_t nblk = (size_t)n[0] * n[1] * n[2] * n[3];
    /* HRR blocks cached by (set, shifts in [-k, k] per centre) */
    const int W = 2 * k + 1;
    size_t ncache = (size_t)NS * W * W * W * W;
    double **cache = (double **)calloc(ncache, sizeof(double *));
    int nm = (int)binom_l(11 + k, k);
    int tup[4] = {0, 0, 0, 0};
    for (int m = 0; m < nm; ++m) {
        /* per centre and direction: derivative count */
        int cnt[4][3];
        memset(cnt, 0, sizeof cnt);
        for (int i = 0; i < k; ++i) cnt[tup[i] / 3][tup[i] % 3]++;
        double *dst = out + (size_t)m * nblk;
        for (int ia = 0; ia < n[0]; ++ia)
            for (int ib = 0; ib < n[1]; ++ib)
                for (int ic = 0; ic < n[2]; ++ic)
                    for (int id = 0; id < n[3]; ++id) {
                        const int *xs[4] = {g_comp[L[0]][ia], g_comp[L[1]][ib], g_comp[L[2]][ic], g_comp[L[3]][id]};
                        /* expansion coefficients per (centre, direction) */
                        double cf[4][3][5];
                        int nt[4][3];
                        for (int cc = 0; cc < 4; ++cc)
                            for (int x = 0; x < 3; ++x) {
                                dexp1(cnt[cc][x], xs[cc][x], cf[cc][x]);
                                nt[cc][x] = cnt[cc][x] + 1;
                            }
                        double val = 0.0;
                        /* iterate over all 12 term indices (mixed radix) */
                        int j[12] = {0};
                        for (;;) {
                            double coef = 1.0;
                            int comp[4][3], raise[4] = {0, 0, 0, 0}, ok = 1;
                            for (int cc = 0; cc < 4 && ok; ++cc)
                                for (int x = 0; x < 3; ++x) {
                                    int jj = j[3 * cc + x];
                                    coef *= cf[cc][x][jj];
                                    comp[cc][x] = xs[cc][x] + 2 * jj - cnt[cc][x];
                                    raise[cc] += jj;
                                    if (comp[cc][x] < 0) ok = 0;
                                }
                            if (ok && coef != 0.0) {
                                int dl[4];
                                for (int cc = 0; cc < 4; ++cc) dl[cc] = comp[cc][0] + comp[cc][1] + comp[cc][2] - L[cc];
                                int srank = set_rank(k, raise);
                                size_t key = ((((size_t)srank * W + dl[0] + k) * W + dl[1] + k) * W + dl[2] + k) * W + dl[3] + k;
                                if (!cache[key]) {
                                    size_t bs = (size_t)ncart(L[0] + dl[0]) * ncart(L[1] + dl[1]) * ncart(L[2] + dl[2]) *
                                                ncart(L[3] + dl[3]);
                                    cache[key] = (double *)malloc(sizeof(double) * bs);
                                    hrr_both(L[0] + dl[0], L[1] + dl[1], L[2] + dl[2], L[3] + dl[3], AB, CD,
                                             S + (size_t)srank * asz, NF, cache[key]);
                                }
                                int nb2 = ncart(L[1] + dl[1]), nc2 = ncart(L[2] + dl[2]), nd2 = ncart(L[3] + dl[3]);
                                size_t o = (((size_t)lidx(comp[0][0], comp[0][1], comp[0][2]) * nb2 +
                                             lidx(comp[1][0], comp[1][1], comp[1][2])) * nc2 +
                                            lidx(comp[2][0], comp[2][1], comp[2][2])) * nd2 +
                                           lidx(comp[3][0], comp[3][1], comp[3][2]);
                                val += coef * cache[key][o];
                            }
                            int p = 0;
                            while (p < 12) {
                                if (++j[p] < nt[p / 3][p % 3]) break;
                                j[p] = 0;
                                ++p;
                            }
                            if (p == 12) break;
                        }
                        dst[(((size_t)ia * n[1] + ib) * n[2] + ic) * n[3] + id] = val;
                    }
        /* next sorted tuple */
        int p = k - 1;
        while (p >= 0 && tup[p] == 11) --p;
        if (p < 0) break;
        tup[p] += 1;
        for (int i = p + 1; i < k; ++i) tup[i] = tup[p];
    }
    for (size_t i = 0; i < ncache; ++i) free(cache[i]);
    free(cache);
    free(v);
    return 0;
}

int qxo_shell_quartet_derivk(const qxo_basis *B, int s1, int s2, int s3, int s4, int k, double *out) {
    init_tables();
    return quartetk(B, s1, s2, s3, s4, k, out);
}

/* Derivative tensor of order k (1..4) with the reference's semantics
 * (eri_deriv_core, libint_interface.cc:2582-2779, and compute_2e_deriv, :1097-1335):
 * slices for the sorted nuclear multi-indices nu_1 <= ... <= nu_k in the order of
 * generate_multi_index_lookup(3N, k); element = sum over the cartesian product of
 * shell positions on each nu_i's atom (direction of nu_i) of the buffer of the
 * sorted centre-direction tuple (libint_interface.cc:1200-1226).  Quartets on one
 * atom are skipped.  slice >= 0 produces that slice only. */
int qxo_eri_derivk(const qxo_basis *B, double thr, int k, long slice, double *out, int nthreads) {
    init_tables();
    if (k < 1 || k > 4) return -1;
    int ns = B->nshell, N3 = 3 * B->natom;
    double *K = (double *)malloc(sizeof(double) * ns * ns);
    double kmax;
    qxo_schwarz(B, K, &kmax, nthreads);
    int *pairs = (int *)malloc(sizeof(int) * ns * (ns + 1));
    int np = qxo_pairs(B, K, kmax, thr, pairs);
    long *s2bf = (long *)malloc(sizeof(long) * ns);
    long n;
    shell2bf_of(B, s2bf, &n);
    size_t n4 = (size_t)n * n * n * n;
    long nslot = binom_l(N3 + k - 1, k);
    long nslice = slice >= 0 ? 1 : nslot;
    memset(out, 0, sizeof(double) * n4 * nslice);
    int *nus = (int *)malloc(sizeof(int) * nslot * k);
    qxo_multi_index_lookup(N3, k, nus);
    int nm = (int)binom_l(11 + k, k);
    double thr2 = thr * thr;
    int lmx = 0;
    for (int s = 0; s < ns; ++s) lmx = B->l[s] > lmx ? B->l[s] : lmx;
    size_t nbmax = (size_t)ncart(lmx) * ncart(lmx) * ncart(lmx) * ncart(lmx);
    int nt = nthreads_of(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double *buf = (double *)malloc(sizeof(double) * nbmax * nm);
#pragma omp for schedule(dynamic)
        for (int ip = 0; ip < np; ++ip) {
            int p1 = pairs[2 * ip], p2 = pairs[2 * ip + 1];
            for (int jp = 0; jp < np; ++jp) {
                int p3 = pairs[2 * jp], p4 = pairs[2 * jp + 1];
                if (K[p1 * ns + p2] * K[p3 * ns + p4] < thr2) continue;
                int at[4] = {B->atom[p1], B->atom[p2], B->atom[p3], B->atom[p4]};
                if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
                quartetk(B, p1, p2, p3, p4, k, buf);
                int nn[4] = {shell_size(B->l[p1]), shell_size(B->l[p2]), shell_size(B->l[p3]), shell_size(B->l[p4])};
                size_t nblk = (size_t)nn[0] * nn[1] * nn[2] * nn[3];
                long b1 = s2bf[p1], b2 = s2bf[p2], b3 = s2bf[p3], b4 = s2bf[p4];
                for (long sl = 0; sl < nslice; ++sl) {
                    long r = slice >= 0 ? slice : sl;
                    const int *nu = nus + r * k;
                    /* choices per derivative operator: positions on its atom */
                    int choice[4][4], nch[4], ok = 1;
                    for (int i = 0; i < k; ++i) {
                        nch[i] = 0;
                        for (int c = 0; c < 4; ++c)
                            if (at[c] == nu[i] / 3) choice[i][nch[i]++] = 3 * c + nu[i] % 3;
                        if (!nch[i]) ok = 0;
                    }
                    if (!ok) continue;
                    /* buffer indices of the cartesian product (sorted) */
                    int bidx[256], nb = 0, pick[4] = {0, 0, 0, 0};
                    for (;;) {
                        int tpl[4];
                        for (int i = 0; i < k; ++i) tpl[i] = choice[i][pick[i]];
                        for (int i = 1; i < k; ++i)
                            for (int q = i; q > 0 && tpl[q - 1] > tpl[q]; --q) { int t = tpl[q]; tpl[q] = tpl[q - 1]; tpl[q - 1] = t; }
                        long rk = 0;
                        int prev = 0;
                        for (int i = 0; i < k; ++i) {
                            for (int x = prev; x < tpl[i]; ++x) rk += binom_l(12 - x + k - i - 2, k - i - 1);
                            prev = tpl[i];
                        }
                        bidx[nb++] = (int)rk;
                        int q = k - 1;
                        while (q >= 0 && ++pick[q] == nch[q]) { pick[q] = 0; --q; }
                        if (q < 0) break;
                    }
                    double *o = out + (size_t)sl * n4;
                    for (int f1 = 0, idx = 0; f1 < nn[0]; ++f1)
                        for (int f2 = 0; f2 < nn[1]; ++f2)
                            for (int f3 = 0; f3 < nn[2]; ++f3)
                                for (int f4 = 0; f4 < nn[3]; ++f4, ++idx) {
                                    double x = 0.0;
                                    for (int t = 0; t < nb; ++t) x += buf[(size_t)bidx[t] * nblk + idx];
                                    long i = b1 + f1, j = b2 + f2, kk = b3 + f3, l = b4 + f4;
                                    o[((i * n + j) * n + kk) * n + l] += x;
                                    if (p1 != p2) o[((j * n + i) * n + kk) * n + l] += x;
                                    if (p3 != p4) o[((i * n + j) * n + l) * n + kk] += x;
                                    if (p1 != p2 && p3 != p4) o[((j * n + i) * n + l) * n + kk] += x;
                                }
                }
            }
        }
        free(buf);
    }
    free(K); free(pairs); free(s2bf); free(nus);
    return 0;
}

/* Index helpers restated from quax/integrals/utils.h:131-172. */
int qxo_how_many_derivs(int k, int n) {
    long val = 1, fact = 1;
    for (int i = 0; i < n; ++i) { val *= 3 * k + i; fact *= i + 1; }
    return (int)(val / fact);
}

/* combinations with repetition of range(nparams) of size order, lexicographic;
 * writes order ints per combination, returns the count. */
int qxo_multi_index_lookup(int nparams, int order, int *out) {
    int cnt = 0;
    int idx[16];
    if (order > 16) return -1;
    for (int i = 0; i < order; ++i) idx[i] = 0;
    if (order == 0) return 1;
    for (;;) {
        for (int i = 0; i < order; ++i) out[cnt * order + i] = idx[i];
        ++cnt;
        int p = order - 1;
        while (p >= 0 && idx[p] == nparams - 1) --p;
        if (p < 0) break;
        idx[p] += 1;
        for (int i = p + 1; i < order; ++i) idx[i] = idx[p];
    }
    return cnt;
}
