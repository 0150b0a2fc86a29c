"""Spherical (pure) basis functions on top of the Cartesian integral engine.

The reference's Libint path is Cartesian (quax/integrals/libint_interface.cc:47-73
calls set_pure(false)); the synthetic workloads with spherical d shells need the
real-solid-harmonic functions.  Every quantity is the Cartesian one transformed
with the block-diagonal matrix T (n_sph x n_cart) of the shells' solid
harmonics:

    G_sph = (T x T x T x T) G_cart          dense tensor: four quarter transforms
                                            (batched GEMMs); unique blocks: one
                                            device kernel per class (qx_cart2sph_block)
    J, K  = T J_cart(T^T D T) T^T,  ...      (J and K are linear in D)
    grad  = grad_cart(T^T D T)              (Gamma built from D factorises)
    S, T, V = T M T^T

so the kernels stay Cartesian and the transforms are FP64 matrix products
(cuBLAS DGEMM, FP64 tensor cores on B200) or, for the unique blocks, a sparse
transform kernel of this library.

Conventions: Cartesian components in Libint's order, normalised so that x^l has
unit norm; spherical functions in Libint's standard order m = -l..l, each of unit
norm (for l = 1: y, z, x).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from ..basis import Basis, cart_components
from . import _lib
from .engine import EriEngine


def _solid_harmonic_monomials(l: int, m: int):
    """{(a, b, c): coefficient} of the real solid harmonic S_lm as a polynomial in
    x, y, z (Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory,
    eqs. 6.4.47-6.4.50: the sum over t, u, v of binomial products, v running over
    half-integers for m < 0), before normalisation."""
    am = abs(m)
    vm = 0.0 if m >= 0 else 0.5
    out = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            v = vm
            while v <= (am / 2.0 - vm) // 1 + vm + 1e-9:
                c = ((-1) ** int(round(t + v - vm)) * 0.25 ** t * math.comb(l, t) * math.comb(l - t, am + t)
                     * math.comb(t, u) * math.comb(am, int(round(2 * v))))
                a = 2 * t + am - int(round(2 * (u + v)))
                b = int(round(2 * (u + v)))
                key = (a, b, l - 2 * t - am)
                out[key] = out.get(key, 0.0) + c
                v += 1.0
    return out


def _dfact(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def cart2sph(l: int) -> np.ndarray:
    """(2l+1, ncart(l)) coefficients of the real solid harmonics (m = -l..l) over
    the Libint-normalised Cartesian components (every component carries the
    normalisation of x^l), each spherical function scaled to unit norm with the
    Cartesian angular overlaps <x^a y^b z^c | x^a' y^b' z^c'> =
    (a+a'-1)!! (b+b'-1)!! (c+c'-1)!! / (2l-1)!!  (zero unless every sum is even)."""
    comps = cart_components(l)
    idx = {c: k for k, c in enumerate(comps)}
    S = np.zeros((len(comps), len(comps)))
    for i, p in enumerate(comps):
        for j, q in enumerate(comps):
            e = [p[k] + q[k] for k in range(3)]
            if all(x % 2 == 0 for x in e):
                S[i, j] = _dfact(e[0] - 1) * _dfact(e[1] - 1) * _dfact(e[2] - 1) / _dfact(2 * l - 1)
    M = np.zeros((2 * l + 1, len(comps)))
    for r, m in enumerate(range(-l, l + 1)):
        for key, c in _solid_harmonic_monomials(l, m).items():
            M[r, idx[key]] += c
        M[r] /= math.sqrt(M[r] @ S @ M[r])
    return M


# T_l for l = 0..3, row-major and concatenated: the coefficient table of the
# device transform (qx_cart2sph_block)
_T_PACKED = np.ascontiguousarray(np.concatenate([cart2sph(l).reshape(-1) for l in range(4)]))


def transform_matrix(basis: Basis) -> np.ndarray:
    """Block-diagonal T (n_sph, n_cart) of a basis."""
    blocks = [cart2sph(s.l) for s in basis.shells]
    ns = sum(b.shape[0] for b in blocks)
    nc = sum(b.shape[1] for b in blocks)
    T = np.zeros((ns, nc))
    r = c = 0
    for b in blocks:
        T[r:r + b.shape[0], c:c + b.shape[1]] = b
        r += b.shape[0]
        c += b.shape[1]
    return T


def _quarter(G: torch.Tensor, T: torch.Tensor, axis: int) -> torch.Tensor:
    """Contract index `axis` of G with T (n_sph, n_cart): one batched GEMM."""
    Gm = torch.movedim(G, axis, -1)
    out = Gm @ T.T
    return torch.movedim(out, -1, axis).contiguous()


class SphericalEngine:
    """Spherical-basis front of EriEngine: the Cartesian twin of the basis runs the
    kernels, results are transformed with T."""

    def __init__(self, basis: Basis, ints_tol: float = 1.0e-14, device=None):
        if not basis.pure:
            raise ValueError("SphericalEngine needs a pure basis")
        cart = Basis(basis.shells, basis.natom, False, basis.name)
        self.cart = EriEngine(cart, ints_tol, device)
        self.device = self.cart.device
        self.T = torch.from_numpy(transform_matrix(basis)).to(self.device)
        self.nbf = self.T.shape[0]
        self.natom = self.cart.natom
        self.basis = basis
        self._unique = None  # (class info, Cartesian and spherical unique buffers)

    def close(self):
        self.cart.close()

    def set_charges(self, Z):
        self.cart.set_charges(Z)

    def autotune(self, **kw):
        self.cart.autotune(**kw)

    def _cart_density(self, D):
        D = D.to(device=self.device, dtype=torch.float64)
        return (self.T.T @ D @ self.T).contiguous()

    # -- two-electron -------------------------------------------------------------
    def eri(self) -> torch.Tensor:
        G = self.cart.eri()
        for ax in range(4):
            G = _quarter(G, self.T, ax)
        return G

    def eri_unique(self):
        """Per class, the spherical blocks of the screened unique quartets:
        {(la,lb,lc,ld): (s_a, s_b, s_c, s_d, nq) tensor} -- the Cartesian unique
        layout transformed class by class on the device (qx_cart2sph_block: one
        thread per spherical value, the non-zero solid-harmonic coefficients
        only), into one buffer kept between calls: the returned views hold the
        latest call's values."""
        if self._unique is None:
            info = [c for c in self.cart.class_info()]
            out_c = torch.empty(self.cart.unique_size(), dtype=torch.float64, device=self.device)
            nsph = sum(int(np.prod([2 * l + 1 for l in c["l"]])) * c["nq"] for c in info)
            out_s = torch.empty(max(nsph, 1), dtype=torch.float64, device=self.device)
            self._unique = (info, out_c, out_s)
        info, out_c, out_s = self._unique
        self.cart.eri_unique(out_c)
        lib = _lib.load()
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        res, base, base_s = {}, 0, 0
        for c in info:
            l4 = tuple(c["l"])
            size = int(np.prod([(l + 1) * (l + 2) // 2 for l in l4])) * c["nq"]
            dims_s = [2 * l + 1 for l in l4]
            size_s = int(np.prod(dims_s)) * c["nq"]
            if c["nq"]:
                la = np.array(l4, dtype=np.int32)
                with torch.cuda.device(self.device):
                    _lib.check(lib.qx_cart2sph_block(C.c_void_p(out_c[base:].data_ptr()),
                                                     C.c_void_p(out_s[base_s:].data_ptr()), _lib.iptr(la),
                                                     c["nq"], _lib.dptr(_T_PACKED), stream), "qx_cart2sph_block")
                res[l4] = out_s[base_s:base_s + size_s].view(*dims_s, c["nq"])
            base += size
            base_s += size_s
        return res

    def eri_unique_gemm(self):
        """eri_unique through four batched-GEMM quarter transforms per class
        (torch/cuBLAS); the check on the device transform."""
        out_c = torch.empty(self.cart.unique_size(), dtype=torch.float64, device=self.device)
        self.cart.eri_unique(out_c)
        res, base = {}, 0
        for c in self.cart.class_info():
            la, lb, lc, ld = c["l"]
            dims = [(l + 1) * (l + 2) // 2 for l in (la, lb, lc, ld)]
            size = int(np.prod(dims)) * c["nq"]
            if c["nq"]:
                blk = out_c[base:base + size].view(*dims, c["nq"])
                for ax, l in enumerate((la, lb, lc, ld)):
                    M = torch.from_numpy(cart2sph(l)).to(self.device)
                    blk = _quarter(blk, M, ax)
                res[(la, lb, lc, ld)] = blk
            base += size
        return res

    def jk(self, D):
        Jc, Kc = self.cart.jk(self._cart_density(D))
        return self.T @ Jc @ self.T.T, self.T @ Kc @ self.T.T

    def grad_adjoint(self, D, cj: float = 1.0, ck: float = -0.5):
        return self.cart.grad_adjoint(self._cart_density(D), cj, ck)

    def grad_adjoint_jvp(self, D, v, cj: float = 1.0, ck: float = -0.5):
        return self.cart.grad_adjoint_jvp(self._cart_density(D), v, cj, ck)

    def eri_deriv(self, deriv_vec) -> torch.Tensor:
        G = self.cart.eri_deriv(deriv_vec)
        for ax in range(4):
            G = _quarter(G, self.T, ax)
        return G

    # -- one-electron -------------------------------------------------------------
    def oei(self):
        return tuple(self.T @ M @ self.T.T for M in self.cart.oei())

    def oei_deriv(self, order: int = 1):
        return tuple(torch.einsum("ai,xij,bj->xab", self.T, M, self.T) for M in self.cart.oei_deriv(order))


def make_engine(basis: Basis, ints_tol: float = 1.0e-14, device=None):
    """EriEngine for a Cartesian basis, SphericalEngine for a pure one."""
    return SphericalEngine(basis, ints_tol, device) if basis.pure else EriEngine(basis, ints_tol, device)
