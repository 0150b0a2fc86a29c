// qx_setup.h -- host-side set-up shared by every entry point that builds the
// device tables of a basis (qx_initialize and qx_compute_2e_int_noalloc):
// shell validation and Libint-convention normalisation, the primitive-pair and
// shell-pair records, and the Boys-function table.
#pragma once
#include <string>
#include <vector>

#include "qx_device.cuh"

namespace qx {

struct ShellTables {
    std::vector<int> l, nprim, atom, poff, bf;
    std::vector<double> alpha, coef;  // normalised contraction coefficients
    int nbf = 0;
};

// Validates the shells (l in [0, lmax], 1..64 primitives, atom index, positive
// finite exponents, finite coefficients, non-degenerate contraction) and
// normalises the contractions so that the x^l component of each contracted shell
// has unit norm (Libint's convention).  Returns QX_OK, or QX_E_INVALID /
// QX_E_UNSUPPORTED with `err` set (prefixed by `who`).
int normalize_shells(const char* who, int natom, int nshell, const int* shell_l, const int* shell_nprim,
                     const int* shell_atom, const double* exps, const double* coefs, int lmax, ShellTables& t,
                     std::string& err);

// Shell pairs s1 >= s2 in the reference's order, each in canonical orientation
// (higher angular momentum first), with their primitive-pair records; pcls is the
// pair class l1 (l1 + 1) / 2 + l2 of each.
void build_pairs(const ShellTables& t, const double* coords, std::vector<PrimPair>& prims,
                 std::vector<PairInfo>& pairs, std::vector<int>& pcls);

// Boys table F_m(T_g) (BOYS_NG x BOYS_NM, row-major [g][m]); built once per
// process on first use.
const std::vector<double>& boys_table();

}  // namespace qx
