// ref_utils_shim.cpp -- builds the reference's own index helpers for parity tests.
//
// TEST INFRASTRUCTURE ONLY.  The reference header quax/integrals/utils.h is
// included from the reference tree at compile time (oracle/build_ref.sh passes its
// path); nothing of it is copied here.  The header also declares helpers that use
// Libint types (get_atoms, make_ao_cabs); the minimal declarations below only let
// those compile -- they are never called.  The extern "C" wrappers expose the
// integer helpers the ERI derivative path depends on:
//   how_many_derivs (utils.h:131-141), generate_multi_index_lookup (utils.h:158-172),
//   process_deriv_vec (utils.h:116-128), cartesian_product (utils.h:100-114).
#include <algorithm>
#include <fstream>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

namespace libint2 {
struct Atom {
    int atomic_number = 0;
    double x = 0, y = 0, z = 0;
};
inline std::vector<Atom> read_dotxyz(std::istream&) { return {}; }
struct Contraction {
    int l = 0;
};
struct Shell {
    std::vector<Contraction> contr{Contraction{}};
};
struct BasisSet {
    BasisSet() = default;
    BasisSet(std::string, const std::vector<Atom>&) {}
    BasisSet(const std::vector<Atom>&, const std::vector<std::vector<Shell>>&) {}
    void set_pure(bool) {}
    std::vector<std::vector<long>> atom2shell(const std::vector<Atom>&) const { return {}; }
    Shell operator[](long) const { return Shell{}; }
};
}  // namespace libint2

#include REF_UTILS_H

extern "C" {

int ref_how_many_derivs(int k, int n) { return how_many_derivs(k, n); }

// writes count*order ints (lexicographic combinations with repetition); returns count
int ref_multi_index_lookup(int nparams, int order, int* out, int cap) {
    auto v = generate_multi_index_lookup(nparams, order);
    int k = 0;
    for (auto& c : v)
        for (int x : c)
            if (k < cap) out[k++] = x;
    return (int)v.size();
}

// deriv_vec -> (atoms[], coords[]); returns the number of entries (the order)
int ref_process_deriv_vec(const int* dv, int len, int* atoms, int* coords) {
    std::vector<int> d(dv, dv + len), a, c;
    process_deriv_vec(d, &a, &c);
    for (size_t i = 0; i < a.size(); ++i) {
        atoms[i] = a[i];
        coords[i] = c[i];
    }
    return (int)a.size();
}

// cartesian product of nsets lists (flattened with sizes); returns the number of
// combinations, each nsets ints, written to out (up to cap ints)
int ref_cartesian_product(const int* flat, const int* sizes, int nsets, int* out, int cap) {
    std::vector<std::vector<int>> v;
    int o = 0;
    for (int i = 0; i < nsets; ++i) {
        v.emplace_back(flat + o, flat + o + sizes[i]);
        o += sizes[i];
    }
    auto r = cartesian_product(v);
    int k = 0;
    for (auto& c : r)
        for (int x : c)
            if (k < cap) out[k++] = x;
    return (int)r.size();
}
}
