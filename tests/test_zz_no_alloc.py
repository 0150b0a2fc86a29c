"""The non-allocating ERI entry point against the regular handle path (GPU).

qx_compute_2e_int_noalloc serves callers that must not have the library call
cudaMalloc: an XLA/JAX custom call (the runtime owns and pre-reserves device
memory), real-time hosts that forbid allocation after start-up, and code that
keeps every device byte in its own pool.  It keeps its tables in one fixed static
device array instead.  This file is collected last so that, if it fails, a run
stopped at the first failure has already run every other test; it also passes on
its own in a fresh process.

Tolerance: 1e-12 absolute per integral, as for every FP64 ERI parity test.
"""
import ctypes

import numpy as np
import pytest
import torch

from quax_b200.basis import Basis, Shell, SyntheticSpec, build_basis, h2o_config1, synthetic_molecule

pytestmark = pytest.mark.gpu
ATOL = 1e-12


def _noalloc(basis, tol, out):
    """Call the entry point through the C ABI; the caller (this test) owns `out`."""
    from quax_b200.integrals import _lib

    lib = _lib.load()
    fl = basis.flat()
    coords = np.ascontiguousarray(basis.atom_coords().reshape(-1))
    rc = lib.qx_compute_2e_int_noalloc(
        basis.natom, _lib.dptr(coords), basis.nshell, _lib.iptr(fl["l"]), _lib.iptr(fl["nprim"]),
        _lib.iptr(fl["atom"]), _lib.dptr(fl["exps"]), _lib.dptr(fl["coefs"]), float(tol),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, lib.qx_last_error().decode()


def _handle_eri(basis, tol):
    from quax_b200.integrals.engine import EriEngine

    eng = EriEngine(basis, tol)
    G = eng.eri().clone()
    eng.close()
    return G


def test_noalloc_matches_handle_path_two_calls():
    # d shells on every atom so the large (cooperative) classes take part
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0, charges=(6, 8))
    b = synthetic_molecule(spec, 11)[1]
    ref = _handle_eri(b, 1e-12)
    n = b.nbf()
    out = torch.full((n, n, n, n), float("nan"), dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row share (and reuse) the static array
        rc, msg = _noalloc(b, 1e-12, out)
        assert rc == 0, msg
        assert torch.isfinite(out).all()
        assert (out - ref).abs().max().item() < ATOL, f"call {call}"


def test_noalloc_after_a_different_basis():
    # the array keeps the previous call's tables; a new basis must overwrite them
    h2o = build_basis(h2o_config1(), "sto-3g")
    out7 = torch.empty((7, 7, 7, 7), dtype=torch.float64, device="cuda")
    rc, msg = _noalloc(h2o, 1e-14, out7)
    assert rc == 0, msg
    assert (out7 - _handle_eri(h2o, 1e-14)).abs().max().item() < ATOL


def test_noalloc_rejects_basis_beyond_the_scratch():
    # 240 shells of 8 primitives: the pair tables alone exceed the 16 MiB array
    rng = np.random.default_rng(3)
    shells = [Shell(0, np.sort(rng.uniform(0.5, 5.0, 8))[::-1].copy(), rng.uniform(0.1, 1.0, 8),
                    np.array([0.0, 0.0, 1.3 * a]), a) for a in range(240)]
    big = Basis(shells, 240)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    rc, msg = _noalloc(big, 1e-12, out)
    assert rc == -1 and "scratch" in msg
