"""Device-resident ERI engine: one C-ABI handle per molecule/basis.

``EriEngine`` owns a ``qx_handle`` (shells, pair data, Schwarz table and the
screened quartet lists live on the GPU) and returns torch tensors on that GPU.
It is the object the reference-shaped ``libint_interface`` module and the
``TEI`` primitives in this package are built on.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ..basis import Basis
from ..utils import how_many_derivs
from . import _lib


def _stream_ptr(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream


class EriEngine:
    def __init__(self, basis: Basis, ints_tol: float = 1.0e-14, device=None):
        if basis.pure:
            raise NotImplementedError("spherical shells are not supported by this engine (Cartesian only; see SphericalEngine)")
        lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.QuaxError("no CUDA device: the ERI engine has no CPU path")
        self.device = torch.device(device if device is not None else f"cuda:{torch.cuda.current_device()}")
        fl = basis.flat()
        self.basis = basis
        self.natom = basis.natom
        coords = np.ascontiguousarray(basis.atom_coords().reshape(-1), dtype=np.float64)
        self._keep = (coords, fl)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(
                lib.qx_initialize(
                    basis.natom, _lib.dptr(coords), basis.nshell, _lib.iptr(fl["l"]), _lib.iptr(fl["nprim"]),
                    _lib.iptr(fl["atom"]), _lib.dptr(fl["exps"]), _lib.dptr(fl["coefs"]), 0, float(ints_tol),
                    C.byref(h),
                ),
                "qx_initialize",
            )
        self._h = h
        self.nbf = lib.qx_nbf(h)
        self.nshell = lib.qx_nshell(h)
        self.ints_tol = ints_tol

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().qx_finalize(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if self._h is None:
            raise _lib.QuaxError("engine was finalized")
        return self._h

    # -- queries --------------------------------------------------------------
    # -- one-electron integrals ---------------------------------------------
    def set_charges(self, Z) -> None:
        """Nuclear charges (natom) for the nuclear-attraction integrals."""
        z = np.ascontiguousarray(np.asarray(Z, dtype=np.float64).reshape(-1))
        if z.size != self.natom:
            raise ValueError(f"{z.size} charges for {self.natom} atoms")
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_set_charges(self.handle, C.c_void_p(z.ctypes.data)), "qx_set_charges")

    def oei(self, stream=None):
        """(S, T, V), each (n, n) on the device."""
        n = self.nbf
        S, T, V = (torch.empty((n, n), dtype=torch.float64, device=self.device) for _ in range(3))
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_oei(self.handle, C.c_void_p(S.data_ptr()), C.c_void_p(T.data_ptr()),
                                          C.c_void_p(V.data_ptr()), C.c_void_p(_stream_ptr(stream))), "qx_oei")
        return S, T, V

    def oei_deriv(self, order: int = 1, stream=None):
        """(dS, dT, dV), each (3N, n, n) on the device."""
        n = self.nbf
        shape = (3 * self.natom, n, n)
        dS, dT, dV = (torch.empty(shape, dtype=torch.float64, device=self.device) for _ in range(3))
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_oei_deriv_core(self.handle, int(order), C.c_void_p(dS.data_ptr()),
                                                     C.c_void_p(dT.data_ptr()), C.c_void_p(dV.data_ptr()),
                                                     C.c_void_p(_stream_ptr(stream))), "qx_oei_deriv_core")
        return dS, dT, dV

    def set_shard(self, rank: int, nranks: int) -> None:
        """Keep a cost-balanced contiguous range of every class's quartets (rank of
        nranks); results of the ranks then sum to the full ones."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_set_shard(self.handle, int(rank), int(nranks)), "qx_set_shard")

    def set_precision(self, f32_bound: float) -> None:
        """Mixed precision: FP32 recurrences for quartets with Schwarz bound below
        f32_bound (0 = all FP64).  Reorders the unique layout."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_set_precision(self.handle, float(f32_bound)), "qx_set_precision")

    def precision_split(self):
        """{"la lb lc ld": (FP64 quartets, all quartets)} of this handle's view."""
        lib = _lib.load()
        return {"%d%d%d%d" % c["l"]: (int(lib.qx_precision_split(self.handle, c["cls"])), c["nq"])
                for c in self.class_info() if c["nq"]}

    def unique_quartets(self) -> int:
        return int(_lib.load().qx_unique_quartets(self.handle))

    def unique_size(self) -> int:
        return int(_lib.load().qx_unique_size(self.handle))

    def schwarz(self):
        K = np.empty((self.nshell, self.nshell))
        kmax = C.c_double()
        _lib.check(_lib.load().qx_schwarz(self.handle, _lib.dptr(K), C.byref(kmax)), "qx_schwarz")
        return K, kmax.value

    def class_info(self):
        """Per angular-momentum class: (la,lb,lc,ld), quartets, primitive quartets,
        plain FLOPs, first-derivative FLOPs."""
        lib = _lib.load()
        out = []
        for c in range(lib.qx_num_classes()):
            l4 = np.zeros(4, dtype=np.int32)
            nq, npq = C.c_longlong(), C.c_longlong()
            f, fd = C.c_double(), C.c_double()
            _lib.check(lib.qx_class_info(self.handle, c, _lib.iptr(l4), C.byref(nq), C.byref(npq), C.byref(f),
                                         C.byref(fd)), "qx_class_info")
            out.append(dict(cls=c, l=tuple(int(x) for x in l4), nq=nq.value, prims=npq.value, flops=f.value,
                            flops_deriv=fd.value))
        return out

    # -- integrals ------------------------------------------------------------
    def eri(self, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Dense (n,n,n,n) FP64 ERI tensor on the device (reference layout)."""
        n = self.nbf
        if out is None:
            out = torch.empty((n, n, n, n), dtype=torch.float64, device=self.device)
        assert out.is_contiguous() and out.dtype == torch.float64 and out.numel() == n**4
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_compute_2e_int(self.handle, C.c_void_p(out.data_ptr()), 1, C.c_void_p(_stream_ptr(stream))),
                "qx_compute_2e_int",
            )
        return out

    def eri_host(self) -> np.ndarray:
        """Dense tensor returned in host memory (the reference's return convention)."""
        n = self.nbf
        out = np.empty(n**4)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_compute_2e_int(self.handle, C.c_void_p(out.ctypes.data), 0, C.c_void_p(0)),
                "qx_compute_2e_int",
            )
        return out

    def eri_unique(self, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.unique_size(), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_eri_unique(self.handle, C.c_void_p(out.data_ptr()), C.c_void_p(_stream_ptr(stream))),
                "qx_eri_unique",
            )
        return out

    def eri_unique_class(self, cls: int, out: torch.Tensor, stream=None) -> torch.Tensor:
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_eri_unique_class(self.handle, int(cls), C.c_void_p(out.data_ptr()),
                                                C.c_void_p(_stream_ptr(stream))),
                "qx_eri_unique_class",
            )
        return out

    ENGINE_NAMES = ("sl", "warp", "coop", "wvrr", "wsplit", "dsplit", "rys")

    def autotune(self, plain: bool = True, deriv: bool = True, stream=None) -> None:
        """Time every engine configuration per class on this molecule and keep the fastest."""
        what = (1 if plain else 0) | (2 if deriv else 0)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_autotune(self.handle, what, C.c_void_p(_stream_ptr(stream))), "qx_autotune")

    def engine_config(self):
        """{"la lb lc ld": (plain engine, param, deriv engine, param)} for the classes with quartets."""
        lib = _lib.load()
        out = {}
        for c in self.class_info():
            if not c["nq"]:
                continue
            cfg = np.zeros(4, dtype=np.int32)
            _lib.check(lib.qx_engine_config(self.handle, c["cls"], C.c_void_p(cfg.ctypes.data)), "qx_engine_config")
            out["%d%d%d%d" % c["l"]] = (self.ENGINE_NAMES[cfg[0]], int(cfg[1]), self.ENGINE_NAMES[cfg[2]], int(cfg[3]))
        return out

    def set_engine(self, cls: int, plain: str | None = None, plain_param: int = 0, deriv: str | None = None,
                   deriv_param: int = 0) -> None:
        """Force the engine of one class (names as in ENGINE_NAMES; None keeps the
        current one).  plain_param: log2 lanes per quartet ("sl") or warps per
        quartet ("warp": 1 or 4); deriv_param: warps per quartet ("warp"), or the
        Rys adjoint gradient's table build ("rys": 0 per-unit for small units, 1
        level-parallel)."""
        pe = -1 if plain is None else self.ENGINE_NAMES.index(plain)
        de = -1 if deriv is None else self.ENGINE_NAMES.index(deriv)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_set_engine(self.handle, int(cls), pe, int(plain_param), de, int(deriv_param)),
                       "qx_set_engine")

    def release_scratch(self) -> None:
        """Free the derivative accumulators the handle keeps between calls (for
        many handles on one device; the next derivative call allocates again)."""
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().qx_release_scratch(self.handle), "qx_release_scratch")

    def set_wait_limit(self, polls: int) -> None:
        """Polls of the bounded waits on the split-mode staging copies (0 makes
        them run out: the host-synchronising calls then raise QuaxError)."""
        _lib.check(_lib.load().qx_set_wait_limit(self.handle, int(polls)), "qx_set_wait_limit")

    def class_quartets(self, cls: int) -> np.ndarray:
        """(nq, 4) canonical shell indices of a class's quartets in list order (the
        order of the unique layout)."""
        nq = next(c["nq"] for c in self.class_info() if c["cls"] == cls)
        out = np.zeros((max(nq, 1), 4), dtype=np.int32)
        _lib.check(_lib.load().qx_class_quartets(self.handle, int(cls), _lib.iptr(out)), "qx_class_quartets")
        return out[:nq]

    def unique_blocks(self, out: torch.Tensor | None = None):
        """{class id: (shells (nq, 4), blocks (nq, ncomp))} from the unique layout."""
        u = self.eri_unique(out)
        res = {}
        base = 0
        for c in self.class_info():
            nq = c["nq"]
            ncomp = int(np.prod([(l + 1) * (l + 2) // 2 for l in c["l"]]))
            if nq:
                blk = u[base:base + nq * ncomp].view(ncomp, nq).T
                res[c["cls"]] = (self.class_quartets(c["cls"]), blk)
            base += nq * ncomp
        return res

    def grad_adjoint_jvp(self, D: torch.Tensor, v, cj: float = 1.0, ck: float = -0.5, stream=None) -> torch.Tensor:
        """Hessian-vector product of sum Gamma G (Gamma from D, fixed) along v (3N)."""
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        v = torch.as_tensor(v, dtype=torch.float64).to(self.device).contiguous().reshape(-1)
        if v.numel() != 3 * self.natom:
            raise ValueError(f"v has {v.numel()} entries, expected {3 * self.natom}")
        out = torch.empty(3 * self.natom, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_grad_adjoint_jvp(self.handle, C.c_void_p(D.data_ptr()), float(cj), float(ck),
                                                C.c_void_p(v.data_ptr()), C.c_void_p(out.data_ptr()), 1,
                                                C.c_void_p(_stream_ptr(stream))),
                "qx_grad_adjoint_jvp",
            )
        return out

    def grad_adjoint_class(self, cls: int, D: torch.Tensor, grad: torch.Tensor, cj: float = 1.0, ck: float = -0.5,
                           stream=None) -> torch.Tensor:
        """Adds one class's adjoint-gradient contribution into grad (3N, device)."""
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_grad_adjoint_class(self.handle, int(cls), C.c_void_p(D.data_ptr()), float(cj),
                                                  float(ck), C.c_void_p(grad.data_ptr()),
                                                  C.c_void_p(_stream_ptr(stream))),
                "qx_grad_adjoint_class",
            )
        return grad

    # -- derivatives ----------------------------------------------------------
    def eri_deriv_core(self, order: int = 1, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Dense derivative tensor on the device, reference layout (nderiv, n, n, n, n):
        nderiv = 3N for order 1, 3N(3N+1)/2 for order 2 (nuclear pairs nu1 <= nu2), and
        in general the combinations with repetition of the 3N coordinates (orders 1-4)."""
        n = self.nbf
        shape = (how_many_derivs(self.natom, int(order)), n, n, n, n)
        if out is None:
            out = torch.empty(shape, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_eri_deriv_core(self.handle, int(order), C.c_void_p(out.data_ptr()), 1,
                                              C.c_void_p(_stream_ptr(stream))),
                "qx_eri_deriv_core",
            )
        return out

    def eri_deriv(self, deriv_vec, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """One (n,n,n,n) derivative slice for an integer deriv_vec of length 3N."""
        dv = np.ascontiguousarray(np.asarray(deriv_vec, dtype=np.int32).reshape(-1))
        n = self.nbf
        if out is None:
            out = torch.empty((n, n, n, n), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_compute_2e_deriv(self.handle, _lib.iptr(dv), dv.size, C.c_void_p(out.data_ptr()), 1,
                                                C.c_void_p(_stream_ptr(stream))),
                "qx_compute_2e_deriv",
            )
        return out

    def grad_adjoint(self, D: torch.Tensor, cj: float = 1.0, ck: float = -0.5, out: torch.Tensor | None = None,
                     stream=None) -> torch.Tensor:
        """sum_ijkl Gamma_ijkl d(ij|kl)/dR with Gamma = cj D_ij D_kl + ck D_ik D_jl (3N vector)."""
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        if out is None:
            out = torch.empty(3 * self.natom, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(
                _lib.load().qx_grad_adjoint(self.handle, C.c_void_p(D.data_ptr()), float(cj), float(ck),
                                            C.c_void_p(out.data_ptr()), 1, C.c_void_p(_stream_ptr(stream))),
                "qx_grad_adjoint",
            )
        return out

    def grad_plain(self, D: torch.Tensor, cj: float = 1.0, ck: float = -0.5, images: bool = True,
                   tile_bytes: int = 2 << 30, stream=None) -> torch.Tensor:
        """The plain FP64 derivative-tensor path for sum Gamma dG/dR (3N vector):
        class by class, tiles of unique quartets have their first-derivative
        integrals materialised as a (3N, tile) tensor -- with images=True every
        distinct image of each integral, i.e. the elements of the reference's
        dense (3N, n^4) tensor -- and then contracted with Gamma in one GEMV per
        tile.  Each derivative quartet is evaluated once.  Tiles hold at most
        tile_bytes of derivative tensor."""
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        M = 3 * self.natom
        width = 8 if images else 1
        info = [c for c in self.class_info() if c["nq"]]
        largest = max((int(np.prod([(l + 1) * (l + 2) // 2 for l in c["l"]])) for c in info), default=1) * width
        emax = max(largest, tile_bytes // (8 * M))  # at least one quartet per tile
        B = torch.empty(M * emax, dtype=torch.float64, device=self.device)
        gam = torch.empty(emax, dtype=torch.float64, device=self.device)
        g = torch.zeros(M, dtype=torch.float64, device=self.device)
        lib = _lib.load()
        sp = C.c_void_p(_stream_ptr(stream))
        with torch.cuda.device(self.device):
            for c in info:
                nq = c["nq"]
                ncomp = int(np.prod([(l + 1) * (l + 2) // 2 for l in c["l"]]))
                qt = max(1, emax // (ncomp * width))
                for q0 in range(0, nq, qt):
                    q1 = min(nq, q0 + qt)
                    E = (q1 - q0) * ncomp * width
                    Bv = B[: M * E].view(M, E)
                    Bv.zero_()
                    _lib.check(lib.qx_deriv_tile(self.handle, c["cls"], q0, q1, int(images),
                                                 C.c_void_p(Bv.data_ptr()), E, sp), "qx_deriv_tile")
                    _lib.check(lib.qx_gamma_tile(self.handle, c["cls"], q0, q1, int(images),
                                                 C.c_void_p(D.data_ptr()), float(cj), float(ck),
                                                 C.c_void_p(gam.data_ptr()), sp), "qx_gamma_tile")
                    g += Bv @ gam[:E]
        return g

    # -- Fock-matrix pieces -----------------------------------------------------
    def jk(self, D: torch.Tensor, J: torch.Tensor | None = None, K: torch.Tensor | None = None, stream=None,
           screen: float = 0.0):
        """Direct J_ij = sum (ij|kl) D_kl and K_ij = sum (ik|jl) D_kl (D symmetric).
        screen > 0 skips quartets whose Schwarz bound times the largest density block
        they touch is below it (for incremental builds from a density change)."""
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        n = self.nbf
        if J is None:
            J = torch.empty((n, n), dtype=torch.float64, device=self.device)
        if K is None:
            K = torch.empty((n, n), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            if screen > 0.0:
                _lib.check(
                    _lib.load().qx_jk_screened(self.handle, C.c_void_p(D.data_ptr()), C.c_void_p(J.data_ptr()),
                                               C.c_void_p(K.data_ptr()), float(screen),
                                               C.c_void_p(_stream_ptr(stream))),
                    "qx_jk_screened",
                )
            else:
                _lib.check(
                    _lib.load().qx_jk(self.handle, C.c_void_p(D.data_ptr()), C.c_void_p(J.data_ptr()),
                                      C.c_void_p(K.data_ptr()), 1, C.c_void_p(_stream_ptr(stream))),
                    "qx_jk",
                )
        return J, K
