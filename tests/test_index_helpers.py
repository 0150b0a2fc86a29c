"""Nuclear-derivative index bookkeeping against the reference.

Pinned two ways: golden vectors produced by the reference's own quax/utils.py
(tests/golden/make_golden.py), and the reference's C++ helpers in
quax/integrals/utils.h compiled from the reference tree (oracle/build_ref.sh, when
that library was built).
"""
import ctypes
import itertools
import json
import os

import numpy as np
import pytest

from quax_b200 import utils as U

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libquax_ref_utils.so")


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "index_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("reference helpers not built (oracle/build_ref.sh needs the reference tree)")
    return ctypes.CDLL(REF_SO)


def test_how_many_derivs_golden(golden):
    for k, n, v in golden["how_many_derivs"]:
        assert U.how_many_derivs(k, n) == v


def test_get_deriv_vec_idx_golden(golden):
    for case in golden["get_deriv_vec_idx"]:
        assert U.get_deriv_vec_idx(case["deriv_vec"]) == case["idx"]


def test_rank_is_position_in_lookup():
    for nparams, order in [(6, 1), (9, 2), (12, 3), (12, 2)]:
        lut = U.generate_multi_index_lookup(nparams, order)
        for i, c in enumerate(lut):
            assert U.multiset_rank(c, nparams) == i


def test_multi_index_lookup_vs_reference(ref, oracle_lib):
    for nparams, order in [(12, 1), (12, 2), (9, 3), (30, 2)]:
        cnt = U.how_many_derivs(0, 0) and len(U.generate_multi_index_lookup(nparams, order))
        buf = (ctypes.c_int * (cnt * order))()
        n = ref.ref_multi_index_lookup(nparams, order, buf, cnt * order)
        assert n == cnt
        r = np.array(list(buf)).reshape(n, order)
        assert np.array_equal(r, np.array(U.generate_multi_index_lookup(nparams, order)))
        assert np.array_equal(r, oracle_lib.multi_index_lookup(nparams, order))


def test_how_many_derivs_vs_reference(ref, oracle_lib):
    for k in range(1, 12):
        for n in range(1, 4):
            assert ref.ref_how_many_derivs(k, n) == U.how_many_derivs(k, n) == oracle_lib.how_many_derivs(k, n)


def test_process_deriv_vec_vs_reference(ref):
    rng = np.random.default_rng(0)
    for _ in range(20):
        dv = rng.integers(0, 3, size=9).astype(np.int32)
        a = (ctypes.c_int * 64)()
        c = (ctypes.c_int * 64)()
        n = ref.ref_process_deriv_vec(dv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 9, a, c)
        atoms, coords = U.process_deriv_vec(dv)
        assert list(a)[:n] == atoms and list(c)[:n] == coords


def test_cartesian_product_vs_reference(ref):
    sets = [[2, 5], [8], [0, 3, 11]]
    flat = np.array(list(itertools.chain(*sets)), dtype=np.int32)
    sizes = np.array([len(s) for s in sets], dtype=np.int32)
    out = (ctypes.c_int * 64)()
    n = ref.ref_cartesian_product(flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 3, out, 64)
    assert np.array(list(out)[: n * 3]).reshape(n, 3).tolist() == U.cartesian_product(sets)
