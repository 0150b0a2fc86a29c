"""ctypes front-end of the CPU FP64 oracle (oracle/eri_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, as the reference results to compare with; never by the
product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Basis(C.Structure):
    _fields_ = [
        ("nshell", C.c_int),
        ("natom", C.c_int),
        ("l", _ip),
        ("nprim", _ip),
        ("atom", _ip),
        ("prim_off", _ip),
        ("center", _dp),
        ("alpha", _dp),
        ("coef", _dp),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.qxo_boys.argtypes = [C.c_int, C.c_double, _dp]
        L.qxo_normalize.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp]
        for name in ("qxo_shell_quartet", "qxo_shell_quartet_deriv1"):
            getattr(L, name).argtypes = [C.POINTER(_Basis), C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.qxo_schwarz.argtypes = [C.POINTER(_Basis), _dp, _dp, C.c_int]
        L.qxo_pairs.argtypes = [C.POINTER(_Basis), _dp, C.c_double, C.c_double, _ip]
        L.qxo_compute_2e_int.argtypes = [C.POINTER(_Basis), C.c_double, _dp, C.c_int]
        L.qxo_eri_deriv1.argtypes = [C.POINTER(_Basis), C.c_double, C.c_int, _dp, C.c_int]
        L.qxo_grad_contract.argtypes = [C.POINTER(_Basis), C.c_double, _dp, C.c_double, C.c_double, _dp, C.c_int]
        L.qxo_unique_sample.restype = C.c_long
        L.qxo_unique_sample.argtypes = [C.POINTER(_Basis), C.c_double, C.c_long, C.c_long, C.c_int, _dp, C.c_double,
                                        _dp, C.c_int]
        L.qxo_count_unique.restype = C.c_long
        L.qxo_count_unique.argtypes = [C.POINTER(_Basis), C.c_double, C.c_int]
        L.qxo_shell_quartet_deriv2.argtypes = [C.POINTER(_Basis), C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.qxo_eri_deriv2.argtypes = [C.POINTER(_Basis), C.c_double, C.c_int, _dp, C.c_int]
        L.qxo_quartet_blocks.argtypes = [C.POINTER(_Basis), _ip, C.c_long, _dp, C.c_int]
        L.qxo_grad_quartets.argtypes = [C.POINTER(_Basis), _ip, C.c_long, _dp, C.c_double, C.c_double, _dp,
                                        C.c_int]
        L.qxo_shell_quartet_derivk.argtypes = [C.POINTER(_Basis), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.qxo_eri_derivk.argtypes = [C.POINTER(_Basis), C.c_double, C.c_int, C.c_long, _dp, C.c_int]
        L.qxo_how_many_derivs.argtypes = [C.c_int, C.c_int]
        L.qxo_multi_index_lookup.argtypes = [C.c_int, C.c_int, _ip]
        _LIB = L
    return _LIB


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class OracleBasis:
    """Holds the flat arrays alive and the C struct pointing at them."""

    def __init__(self, basis):
        if basis.pure:
            raise ValueError("the oracle works in the Cartesian basis; apply the spherical transform outside")
        fl = basis.flat()
        self.natom = basis.natom
        self.l = fl["l"].astype(np.int32)
        self.nprim = fl["nprim"].astype(np.int32)
        self.atom = fl["atom"].astype(np.int32)
        self.off = fl["prim_off"].astype(np.int32)
        self.center = np.ascontiguousarray(fl["centers"].reshape(-1))
        self.alpha = np.ascontiguousarray(fl["exps"])
        self.coef = np.empty_like(self.alpha)
        L = lib()
        for s in range(len(self.l)):
            o, k = int(self.off[s]), int(self.nprim[s])
            a = np.ascontiguousarray(self.alpha[o : o + k])
            cin = np.ascontiguousarray(fl["coefs"][o : o + k])
            cout = np.empty(k)
            if L.qxo_normalize(int(self.l[s]), k, _p(a), _p(cin), _p(cout)) != 0:
                raise ValueError("non-positive exponent or degenerate contraction")
            self.coef[o : o + k] = cout
        self.s = _Basis(
            len(self.l), basis.natom, _p(self.l, _ip), _p(self.nprim, _ip), _p(self.atom, _ip), _p(self.off, _ip),
            _p(self.center), _p(self.alpha), _p(self.coef),
        )
        self.nbf = int(sum((l + 1) * (l + 2) // 2 for l in self.l))

    @property
    def ref(self):
        return C.byref(self.s)


def boys(mmax: int, T: float) -> np.ndarray:
    out = np.empty(mmax + 1)
    lib().qxo_boys(mmax, float(T), _p(out))
    return out


def shell_quartet(ob: OracleBasis, s1, s2, s3, s4, deriv=False) -> np.ndarray:
    n = [(int(ob.l[s]) + 1) * (int(ob.l[s]) + 2) // 2 for s in (s1, s2, s3, s4)]
    if deriv:
        out = np.empty((12,) + tuple(n))
        lib().qxo_shell_quartet_deriv1(ob.ref, s1, s2, s3, s4, _p(out))
    else:
        out = np.empty(tuple(n))
        lib().qxo_shell_quartet(ob.ref, s1, s2, s3, s4, _p(out))
    return out


def schwarz(ob: OracleBasis, nthreads: int = 0):
    ns = len(ob.l)
    K = np.empty((ns, ns))
    kmax = C.c_double()
    lib().qxo_schwarz(ob.ref, _p(K), C.byref(kmax), nthreads)
    return K, kmax.value


def pairs(ob: OracleBasis, thr: float, nthreads: int = 0) -> np.ndarray:
    K, kmax = schwarz(ob, nthreads)
    ns = len(ob.l)
    out = np.empty(ns * (ns + 1), dtype=np.int32)
    n = lib().qxo_pairs(ob.ref, _p(K), kmax, thr, _p(out, _ip))
    return out[: 2 * n].reshape(n, 2)


def compute_2e_int(ob: OracleBasis, thr: float, nthreads: int = 0) -> np.ndarray:
    n = ob.nbf
    out = np.empty((n, n, n, n))
    lib().qxo_compute_2e_int(ob.ref, thr, _p(out), nthreads)
    return out


def eri_deriv1(ob: OracleBasis, thr: float, deriv_idx: int = -1, nthreads: int = 0) -> np.ndarray:
    n = ob.nbf
    shape = (n, n, n, n) if deriv_idx >= 0 else (3 * ob.natom, n, n, n, n)
    out = np.empty(shape)
    lib().qxo_eri_deriv1(ob.ref, thr, int(deriv_idx), _p(out), nthreads)
    return out


def shell_quartet_deriv2(ob: OracleBasis, s1, s2, s3, s4) -> np.ndarray:
    """(12, 12, n1, n2, n3, n4) second-derivative blocks, index 3*centre + xyz."""
    n = [(int(ob.l[s]) + 1) * (int(ob.l[s]) + 2) // 2 for s in (s1, s2, s3, s4)]
    out = np.empty((12, 12) + tuple(n))
    lib().qxo_shell_quartet_deriv2(ob.ref, s1, s2, s3, s4, _p(out))
    return out


def eri_deriv2(ob: OracleBasis, thr: float, pair_idx: int = -1, nthreads: int = 0) -> np.ndarray:
    """Second-derivative tensor (3N(3N+1)/2, n, n, n, n), reference semantics."""
    n = ob.nbf
    N3 = 3 * ob.natom
    shape = (n, n, n, n) if pair_idx >= 0 else (N3 * (N3 + 1) // 2, n, n, n, n)
    out = np.empty(shape)
    lib().qxo_eri_deriv2(ob.ref, thr, int(pair_idx), _p(out), nthreads)
    return out


def quartet_blocks(ob: OracleBasis, shells: np.ndarray, nthreads: int = 0) -> np.ndarray:
    """(nq, nblk) contracted blocks of a list of shell quartets of one class
    (shells: (nq, 4) shell indices, in that centre order)."""
    q4 = np.ascontiguousarray(np.asarray(shells, dtype=np.int32).reshape(-1, 4))
    if q4.shape[0] == 0:
        return np.zeros((0, 0))
    nblk = int(np.prod([(int(ob.l[s]) + 1) * (int(ob.l[s]) + 2) // 2 for s in q4[0]]))
    out = np.empty((q4.shape[0], nblk))
    if lib().qxo_quartet_blocks(ob.ref, _p(q4, _ip), q4.shape[0], _p(out), nthreads) != 0:
        raise ValueError("quartet_blocks: the quartets are not of one class")
    return out


def grad_quartets(ob: OracleBasis, shells: np.ndarray, D: np.ndarray, cj=1.0, ck=-0.5, nthreads: int = 0):
    """Adjoint-gradient contribution (3N) of a list of 8-fold-unique quartets."""
    q4 = np.ascontiguousarray(np.asarray(shells, dtype=np.int32).reshape(-1, 4))
    D = np.ascontiguousarray(D, dtype=np.float64)
    g = np.zeros(3 * ob.natom)
    lib().qxo_grad_quartets(ob.ref, _p(q4, _ip), q4.shape[0], _p(D), float(cj), float(ck), _p(g), nthreads)
    return g


def shell_quartet_derivk(ob: OracleBasis, s1, s2, s3, s4, k: int) -> np.ndarray:
    """(C(11+k, k), n1, n2, n3, n4) derivative blocks of order k, all four centres
    direct, indexed by the sorted k-tuples of centre-directions 3*centre + xyz."""
    from math import comb

    n = [(int(ob.l[s]) + 1) * (int(ob.l[s]) + 2) // 2 for s in (s1, s2, s3, s4)]
    out = np.empty((comb(11 + k, k),) + tuple(n))
    if lib().qxo_shell_quartet_derivk(ob.ref, s1, s2, s3, s4, int(k), _p(out)) != 0:
        raise ValueError("derivative order must be 1..4")
    return out


def eri_derivk(ob: OracleBasis, thr: float, k: int, slice_idx: int = -1, nthreads: int = 0) -> np.ndarray:
    """Order-k derivative tensor (C(3N+k-1, k), n, n, n, n), reference semantics; one
    slice when slice_idx >= 0."""
    from math import comb

    n = ob.nbf
    N3 = 3 * ob.natom
    shape = (n, n, n, n) if slice_idx >= 0 else (comb(N3 + k - 1, k), n, n, n, n)
    out = np.empty(shape)
    if lib().qxo_eri_derivk(ob.ref, thr, int(k), int(slice_idx), _p(out), nthreads) != 0:
        raise ValueError("derivative order must be 1..4")
    return out


def grad_contract(ob: OracleBasis, thr: float, D: np.ndarray, cj=1.0, ck=-0.5, nthreads: int = 0) -> np.ndarray:
    D = np.ascontiguousarray(D, dtype=np.float64)
    g = np.empty(3 * ob.natom)
    lib().qxo_grad_contract(ob.ref, thr, _p(D), cj, ck, _p(g), nthreads)
    return g


def unique_sample(ob: OracleBasis, thr: float, stride: int, phase: int = 0, deriv=False, nthreads: int = 0,
                  K=None, kmax: float = 0.0):
    """Evaluate every stride-th screened unique quartet; K/kmax from schwarz() skip the
    screening pass so only quartet work is timed."""
    cs = C.c_double()
    Kp = _p(np.ascontiguousarray(K, dtype=np.float64)) if K is not None else None
    n = lib().qxo_unique_sample(ob.ref, thr, int(stride), int(phase), int(bool(deriv)), Kp, float(kmax), C.byref(cs),
                                nthreads)
    return n, cs.value


def count_unique(ob: OracleBasis, thr: float, nthreads: int = 0) -> int:
    return int(lib().qxo_count_unique(ob.ref, thr, nthreads))


def how_many_derivs(k: int, n: int) -> int:
    return int(lib().qxo_how_many_derivs(k, n))


def multi_index_lookup(nparams: int, order: int) -> np.ndarray:
    cnt = how_many_derivs(0, 0)  # placeholder to load lib
    from math import comb

    cnt = comb(nparams + order - 1, order)
    out = np.empty(max(cnt * order, 1), dtype=np.int32)
    n = lib().qxo_multi_index_lookup(nparams, order, _p(out, _ip))
    return out[: n * order].reshape(n, order)
