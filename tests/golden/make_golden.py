"""Generates tests/golden/index_golden.json from the reference's own Python helpers.

Run as `python make_golden.py REFERENCE_ROOT` (or with $QUAX_REFERENCE set) where the
reference tree is available: it loads quax/utils.py directly by
path (that module needs only numpy and itertools; the quax package itself needs jax
and psi4, which are absent), evaluates how_many_derivs and get_deriv_vec_idx on a
fixed set of cases, and writes the results.  Test infrastructure only.
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None  # the reference tree: first argument, or $QUAX_REFERENCE


def load_ref_utils():
    spec = importlib.util.spec_from_file_location("quax_ref_utils", os.path.join(REF, "quax", "utils.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QUAX_REFERENCE")
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: make_golden.py REFERENCE_ROOT  (or set QUAX_REFERENCE)")
    ru = load_ref_utils()
    hm = [[k, n, int(ru.how_many_derivs(k, n))] for k in range(1, 7) for n in range(1, 4)]
    rng = np.random.default_rng(2024)
    cases = []
    for natom in (1, 2, 3, 4):
        ncart = 3 * natom
        for order in (1, 2, 3):
            seen = set()
            for _ in range(12):
                dv = np.zeros(ncart, dtype=int)
                for i in rng.integers(0, ncart, size=order):
                    dv[i] += 1
                key = tuple(dv)
                if key in seen:
                    continue
                seen.add(key)
                cases.append({"deriv_vec": dv.tolist(), "idx": int(ru.get_deriv_vec_idx(dv))})
    out = {"source": "reference quax/utils.py (how_many_derivs, get_deriv_vec_idx)",
           "how_many_derivs": hm, "get_deriv_vec_idx": cases}
    with open(os.path.join(HERE, "index_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(hm)} how_many_derivs and {len(cases)} get_deriv_vec_idx cases")


if __name__ == "__main__":
    sys.exit(main())
