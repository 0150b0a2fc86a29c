"""The non-allocating ERI entry point against the regular handle path (GPU).

qx_compute_2e_int_noalloc serves callers that must not have the library call
cudaMalloc: an XLA/JAX custom call (the runtime owns and pre-reserves device
memory), real-time hosts that forbid allocation after start-up, and code that
keeps every device byte in its own pool.  It keeps its tables in one fixed static
device array instead.  This file is collected last so that, if it fails, a run
stopped at the first failure has already run every other test; it also passes on
its own in a fresh process.

Tolerance: 1e-12 absolute per integral, as for every FP64 ERI parity test, against
the handle path and against the CPU oracle.  The property the entry point exists
for -- it allocates no device memory -- is checked with cudaMemGetInfo around a
repeated call and around a call on a new basis.
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


def test_noalloc_matches_handle_path_two_calls(oracle_lib):
    # d shells on every atom so the large (cooperative) classes take part
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0, charges=(6, 8))
    b = synthetic_molecule(spec, 11)[1]
    ref = _handle_eri(b, 1e-12)
    oracle = torch.from_numpy(oracle_lib.compute_2e_int(oracle_lib.OracleBasis(b), 1e-12)).cuda()
    n = b.nbf()
    out = torch.full((n, n, n, n), float("nan"), dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row share (and reuse) the static array
        rc, msg = _noalloc(b, 1e-12, out)
        assert rc == 0, msg
        assert torch.isfinite(out).all()
        assert (out - ref).abs().max().item() < ATOL, f"call {call}"
        assert (out - oracle).abs().max().item() < ATOL, f"call {call}"


def test_noalloc_allocates_no_device_memory():
    """After a first call (which sets the device up and lets the driver load the
    kernels it uses), a repeated call and a call on a new basis -- the same shells
    at displaced positions, so new tables through the same kernels -- leave the
    device's free memory unchanged."""
    spec = SyntheticSpec(natom=3, box=5.0, min_sep=1.2, kmax=3, exp_lo=0.1, exp_hi=50.0)
    b1 = synthetic_molecule(spec, 2)[1]
    b2 = b1.with_coords(b1.atom_coords() + np.random.default_rng(0).normal(0.0, 0.05, size=(b1.natom, 3)))
    n = b1.nbf()
    o1 = torch.empty((n, n, n, n), dtype=torch.float64, device="cuda")
    o2 = torch.empty((n, n, n, n), dtype=torch.float64, device="cuda")
    assert _noalloc(b1, 1e-12, o1)[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _noalloc(b1, 1e-12, o1)[0] == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert _noalloc(b2, 1e-12, o2)[0] == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert (o1 - o2).abs().max().item() > 0.0  # the new basis really gave new integrals


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


def test_noalloc_refuses_stream_capture():
    """The call synchronises (it reads the Schwarz values back), so on a stream
    that is capturing it returns an error instead of breaking the capture."""
    b = build_basis(h2o_config1(), "sto-3g")
    out = torch.empty((7, 7, 7, 7), dtype=torch.float64, device="cuda")
    assert _noalloc(b, 1e-14, out)[0] == 0  # device set-up happens outside the capture
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    res = []
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            res.append(_noalloc(b, 1e-14, out))
    rc, msg = res[0]
    assert rc == -1 and "capturing" in msg
    # (last in the file: a capture left open by a failure here cannot reach
    # another test)
