"""The Rys engine's arithmetic on the CPU (no GPU needed).

tests/rys_host/rys_host.cu compiles the engine's per-primitive functions
(quax_b200/csrc/qx_rys.cuh) for the host and runs them with one thread; the
results are compared with the oracle on random shell quartets of ten classes up
to (ff|ff): the plain block, and the nine first-derivative sums of the adjoint
gradient (dA, dB, dC contracted with a random Gamma), with the level-parallel
table build, the per-unit build, and the compiled kernel's own choice and root
batching; and, up to (ff|df), the derivative blocks of orders 1 and 2 and the
Hessian-vector sums along a random direction.  Tolerances: 1e-11 (plain) and
1e-10 (gradient sums, derivative blocks, Hessian-vector sums), relative to
max(1, largest |value|) -- the oracle's own rounding on the (ff|ff) quartets is
~1e-13 relative -- and the three builds agree with each other to 1e-13.
"""
import ctypes as C
import itertools
import os
import shutil
import subprocess

import numpy as np
import pytest

from quax_b200.basis import Basis, Shell

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
_dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc is not available")
    out = str(tmp_path_factory.mktemp("rys_host") / "librys_host.so")
    cmd = [nvcc, "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "quax_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
           os.path.join(HERE, "rys_host", "rys_host.cu"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lib = C.CDLL(out)
    lib.rys_host.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _ip, _dp, _dp, _dp, _dp, _dp]
    return lib


def _ncart(l):
    return (l + 1) * (l + 2) // 2


def _quartet(oracle_lib, l4, seed):
    """Four shells on four random centres (K 1-2, exponents log-uniform 0.1-20)."""
    rng = np.random.default_rng(seed)
    shells = []
    for c in range(4):
        k = int(rng.integers(1, 3))
        e = np.sort(np.exp(rng.uniform(np.log(0.1), np.log(20.0), size=k)))[::-1].copy()
        shells.append(Shell(int(l4[c]), e, rng.uniform(0.1, 1.0, size=k), rng.uniform(0.0, 3.0, size=3), c))
    ob = oracle_lib.OracleBasis(Basis(shells, 4, False))
    cen = np.ascontiguousarray(np.concatenate([s.center for s in shells]))
    npr = np.array([s.nprim for s in shells], dtype=np.int32)
    ex = np.ascontiguousarray(np.concatenate([s.exps for s in shells]))
    w = np.ascontiguousarray(ob.coef.copy())  # normalised, in shell order
    return ob, cen, npr, ex, w


def _run(lib, kind, cls, build, q, gam, nout, w9=None):
    _, cen, npr, ex, w = q
    out = np.zeros(nout)
    g = np.ascontiguousarray(gam)
    v = np.ascontiguousarray(np.zeros(9) if w9 is None else w9)
    rc = lib.rys_host(kind, cls, build, cen.ctypes.data_as(_dp), npr.ctypes.data_as(_ip), ex.ctypes.data_as(_dp),
                      w.ctypes.data_as(_dp), g.ctypes.data_as(_dp), v.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
    assert rc == 0
    return out


@pytest.mark.parametrize("cls", range(10))
def test_rys_phases_against_oracle(host_lib, oracle_lib, cls):
    l4 = np.zeros(4, dtype=np.int32)
    host_lib.rys_host_class(cls, l4.ctypes.data_as(_ip))
    ncomp = int(np.prod([_ncart(int(l)) for l in l4]))
    q = _quartet(oracle_lib, l4, 100 + cls)
    ob = q[0]
    ref = oracle_lib.shell_quartet(ob, 0, 1, 2, 3).reshape(-1)
    ref1 = oracle_lib.shell_quartet(ob, 0, 1, 2, 3, deriv=True).reshape(12, -1)
    gam = np.random.default_rng(cls).normal(size=ncomp)
    gref = ref1[:9] @ gam
    plain = [_run(host_lib, 0, cls, b, q, np.zeros(1), ncomp) for b in range(3)]
    grad = [_run(host_lib, 1, cls, b, q, gam, 9) for b in range(3)]
    sp, sg = max(1.0, np.abs(ref).max()), max(1.0, np.abs(gref).max())
    for b in range(3):
        assert np.abs(plain[b] - ref).max() < 1e-11 * sp, (tuple(l4), b)
        assert np.abs(grad[b] - gref).max() < 1e-10 * sg, (tuple(l4), b)
        assert np.abs(plain[b] - plain[0]).max() < 1e-13 * sp
        assert np.abs(grad[b] - grad[0]).max() < 1e-13 * sg


@pytest.mark.parametrize("cls", range(8))
def test_rys_derivative_kinds_against_oracle(host_lib, oracle_lib, cls):
    """Orders 1 and 2 (every sorted multi-index of the 12 centre-directions) and
    the Hessian-vector sums h[3X + x] = sum Gamma sum_V w_V d2/dX_x dV, against
    the oracle's first- and second-derivative blocks."""
    l4 = np.zeros(4, dtype=np.int32)
    host_lib.rys_host_class(cls, l4.ctypes.data_as(_ip))
    ncomp = int(np.prod([_ncart(int(l)) for l in l4]))
    q = _quartet(oracle_lib, l4, 200 + cls)
    ob = q[0]
    ref1 = oracle_lib.shell_quartet(ob, 0, 1, 2, 3, deriv=True).reshape(12, -1)
    ref2 = oracle_lib.shell_quartet_deriv2(ob, 0, 1, 2, 3).reshape(12, 12, -1)
    pairs = list(itertools.combinations_with_replacement(range(12), 2))
    r2 = np.stack([ref2[a, b] for a, b in pairs])
    rng = np.random.default_rng(cls)
    gam, w9 = rng.normal(size=ncomp), rng.normal(size=9)
    href = np.array([sum(w9[v] * (ref2[p, v] @ gam) for v in range(9)) for p in range(9)])
    for b in range(3):
        d1 = _run(host_lib, 11, cls, b, q, np.zeros(1), 12 * ncomp).reshape(12, -1)
        assert np.abs(d1 - ref1).max() < 1e-10 * max(1.0, np.abs(ref1).max()), (tuple(l4), b)
        d2 = _run(host_lib, 12, cls, b, q, np.zeros(1), len(pairs) * ncomp).reshape(len(pairs), -1)
        assert np.abs(d2 - r2).max() < 1e-10 * max(1.0, np.abs(r2).max()), (tuple(l4), b)
        h = _run(host_lib, 2, cls, b, q, gam, 9, w9)
        assert np.abs(h - href).max() < 1e-10 * max(1.0, np.abs(href).max()), (tuple(l4), b)
