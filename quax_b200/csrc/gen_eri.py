#!/usr/bin/env python3
"""Generator of the per-class Obara-Saika / Head-Gordon-Pople device code.

Emits ``gen/eri_classes.cuh``: one ``EriCls<LA,LB,LC,LD>`` and one
``DerCls<LA,LB,LC,LD>`` specialisation per canonical angular-momentum class
(LA>=LB, LC>=LD, (LA,LB) >= (LC,LD) in pair-class order).  Every recurrence step
is emitted as straight-line FP64 code over named scalars, pruned to the values
the class actually needs, so nvcc sees SSA values rather than an indexed array.

Method (published mathematics, written here from the papers):
  * VRR  -- Obara & Saika, J. Chem. Phys. 84, 3963 (1986), eq. (39) restricted
    to [e0|f0]^(m) (b = d = 0) as in Head-Gordon & Pople, J. Chem. Phys. 89,
    5777 (1988):
      [e+1_i,0|00]^(m) = PA_i[e0|00]^(m) + WP_i[e0|00]^(m+1)
                       + e_i/(2z) ([e-1_i,0|00]^(m) - rho/z [e-1_i,0|00]^(m+1))
      [e0|f+1_j,0]^(m) = QC_j[e0|f0]^(m) + WQ_j[e0|f0]^(m+1)
                       + f_j/(2h) ([e0|f-1_j,0]^(m) - rho/h [e0|f-1_j,0]^(m+1))
                       + e_j/(2(z+h)) [e-1_j,0|f0]^(m+1)
  * HRR  -- Head-Gordon & Pople: (a,b+1_i| = (a+1_i,b| + AB_i (a,b|, and the ket
    analogue, applied once per contracted quartet.
  * First derivatives -- d/dA_i g_a = 2 alpha g_{a+1_i} - a_i g_{a-1_i}; the
    2alpha / 2beta / 2gamma weights are folded into separate primitive
    accumulators, the D-centre derivative follows from translational invariance.

Run:  python gen_eri.py [LMAX]   (default LMAX=2)
"""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Tuple

Trip = Tuple[int, int, int]


def comps(l: int) -> List[Trip]:
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def ncart(l):
    return (l + 1) * (l + 2) // 2


def hoff(l):
    return l * (l + 1) * (l + 2) // 6


def lidx(t: Trip) -> int:
    k = t[1] + t[2]
    return k * (k + 1) // 2 + t[2]


def gidx(t: Trip) -> int:
    return hoff(sum(t)) + lidx(t)


def sh(t: Trip, i: int, s: int) -> Trip:
    y = list(t)
    y[i] += s
    return tuple(y)


def first_dir(t: Trip) -> int:
    return 0 if t[0] > 0 else (1 if t[1] > 0 else 2)


XYZ = "xyz"


class Emitter:
    """SSA emitter.  ctype is the value type (the warp programs use the template
    parameter T, so one program serves FP64 and FP32 recurrences); lit formats a
    constant of that type."""

    def __init__(self, prefix: str, ctype: str = "double"):
        self.lines: List[str] = []
        self.n = 0
        self.prefix = prefix
        self.ctype = ctype

    def lit(self, x: float) -> str:
        return repr(float(x)) if self.ctype == "double" else f"{self.ctype}({float(x)!r})"

    def new(self, expr: str) -> str:
        name = f"{self.prefix}{self.n}"
        self.n += 1
        self.lines.append(f"const {self.ctype} {name} = {expr};")
        return name


class VRR:
    """Demand-driven VRR DAG over (e, f, m); leaves pref*F_m held in Fp[m]."""

    def __init__(self, em: Emitter):
        self.em = em
        self.memo: Dict[Tuple[Trip, Trip, int], str] = {}

    def get(self, e: Trip, f: Trip, m: int) -> str:
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        if sum(e) == 0 and sum(f) == 0:
            name = f"Fp[{m}]"
        elif sum(f) == 0:
            i = first_dir(e)
            n = e[i]
            em1 = sh(e, i, -1)
            terms = [f"q.PA{XYZ[i]} * {self.get(em1, f, m)}", f"q.WP{XYZ[i]} * {self.get(em1, f, m + 1)}"]
            if n >= 2:
                em2 = sh(e, i, -2)
                terms.append(
                    f"{self.em.lit(n - 1)} * q.oo2z * ({self.get(em2, f, m)} - q.roz * {self.get(em2, f, m + 1)})"
                )
            name = self.em.new(" + ".join(terms))
        else:
            j = first_dir(f)
            nf = f[j]
            fm1 = sh(f, j, -1)
            terms = [f"q.QC{XYZ[j]} * {self.get(e, fm1, m)}", f"q.WQ{XYZ[j]} * {self.get(e, fm1, m + 1)}"]
            if nf >= 2:
                fm2 = sh(f, j, -2)
                terms.append(
                    f"{self.em.lit(nf - 1)} * q.oo2e * ({self.get(e, fm2, m)} - q.roe * {self.get(e, fm2, m + 1)})"
                )
            if e[j] >= 1:
                terms.append(f"{self.em.lit(e[j])} * q.oo2ze * {self.get(sh(e, j, -1), fm1, m + 1)}")
            name = self.em.new(" + ".join(terms))
        self.memo[key] = name
        return name


class AccSpace:
    """Accumulator layout: e in [elo, ehi], f in [flo, fhi] (global Cartesian index)."""

    def __init__(self, name: str, elo, ehi, flo, fhi):
        self.name = name
        self.elo, self.ehi, self.flo, self.fhi = max(elo, 0), ehi, max(flo, 0), fhi
        self.ne = hoff(self.ehi + 1) - hoff(self.elo)
        self.nf = hoff(self.fhi + 1) - hoff(self.flo)
        self.size = self.ne * self.nf

    def index(self, e: Trip, f: Trip) -> int:
        return (gidx(e) - hoff(self.elo)) * self.nf + (gidx(f) - hoff(self.flo))

    def targets(self):
        for le in range(self.elo, self.ehi + 1):
            for e in comps(le):
                for lf in range(self.flo, self.fhi + 1):
                    for f in comps(lf):
                        yield e, f


class HRR:
    """HRR DAG over one accumulator space: ket first (reduce d), then bra."""

    def __init__(self, em: Emitter, acc: AccSpace):
        self.em = em
        self.acc = acc
        self.memo: Dict[Tuple[Trip, Trip, Trip, Trip], str] = {}

    def get(self, a: Trip, b: Trip, c: Trip, d: Trip) -> str:
        key = (a, b, c, d)
        if key in self.memo:
            return self.memo[key]
        if sum(d) > 0:
            j = first_dir(d)
            x = self.get(a, b, sh(c, j, 1), sh(d, j, -1))
            y = self.get(a, b, c, sh(d, j, -1))
            name = self.em.new(f"{x} + CD{XYZ[j]} * {y}")
        elif sum(b) > 0:
            i = first_dir(b)
            x = self.get(sh(a, i, 1), sh(b, i, -1), c, d)
            y = self.get(a, sh(b, i, -1), c, d)
            name = self.em.new(f"{x} + AB{XYZ[i]} * {y}")
        else:
            name = f"{self.acc.name}({self.acc.index(a, c)})"
        self.memo[key] = name
        return name


def gen_plain(la, lb, lc, ld) -> str:
    lab, lcd = la + lb, lc + ld
    S = lab + lcd
    acc = AccSpace("acc", la, lab, lc, lcd)
    out: List[str] = []
    out.append(f"template <> struct EriCls<{la}, {lb}, {lc}, {ld}> {{")
    out.append(f"  static constexpr int S = {S};")
    out.append(f"  static constexpr int NACC = {acc.size};")
    out.append(f"  static constexpr int NOUT = {ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)};")
    # VRR + accumulate
    em = Emitter("v")
    vr = VRR(em)
    # highest bra AM first: measured to give the smallest peak of live values
    for e, f in reversed(list(acc.targets())):
        v = vr.get(e, f, 0)
        em.lines.append(f"acc({acc.index(e, f)}) += {v};")
    out.append("  template <class Acc, class Q>")
    out.append(
        "  static __device__ __forceinline__ void vrr(Acc& acc, const double* __restrict__ Fp, const Q& q) {"
    )
    out += ["    " + ln for ln in em.lines]
    out.append("  }")
    # HRR (each output stored as soon as it is formed)
    em2 = Emitter("h")
    hr = HRR(em2, acc)
    k = 0
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    v = hr.get(a, b, c, d)
                    em2.lines.append(f"st({k}, {v});")
                    k += 1
    out.append("  template <class Acc, class St>")
    out.append(
        "  static __device__ __forceinline__ void hrr(Acc& acc, St& st,"
        " double ABx, double ABy, double ABz, double CDx, double CDy, double CDz) {"
    )
    out.append("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    out += ["    " + ln for ln in em2.lines]
    out.append("  }")
    out.append("};")
    return "\n".join(out)


def gen_deriv(la, lb, lc, ld) -> str:
    """First-derivative class: 4 accumulators (U, 2a*, 2b*, 2c*) and a hrr that
    writes 9 blocks (A_xyz, B_xyz, C_xyz); D follows by invariance."""
    lab, lcd = la + lb, lc + ld
    S = lab + lcd + 1
    U = AccSpace("U", la - 1, lab, lc - 1, lcd)
    WA = AccSpace("WA", la + 1, lab + 1, lc, lcd)
    WB = AccSpace("WB", la, lab + 1, lc, lcd)
    WC = AccSpace("WC", la, lab, lc + 1, lcd + 1)
    nout = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    out: List[str] = []
    out.append(f"template <> struct DerCls<{la}, {lb}, {lc}, {ld}> {{")
    out.append(f"  static constexpr int S = {S};")
    out.append(f"  static constexpr int NU = {U.size}, NA = {WA.size}, NB = {WB.size}, NC = {WC.size};")
    out.append(f"  static constexpr int NOUT = {nout};")
    em = Emitter("v")
    vr = VRR(em)
    acc_lines = []
    # group by VRR value so each value is loaded once and feeds every set using it
    uses: Dict[Tuple[Trip, Trip], List[str]] = {}
    for sp, w in ((U, None), (WA, "a2"), (WB, "b2"), (WC, "c2")):
        for e, f in sp.targets():
            uses.setdefault((e, f), []).append((sp, w))
    for (e, f), lst in uses.items():
        v = vr.get(e, f, 0)
        for sp, w in lst:
            if w is None:
                acc_lines.append(f"{sp.name}[{sp.index(e, f)}] += {v};")
            else:
                acc_lines.append(f"{sp.name}[{sp.index(e, f)}] = fma({w}, {v}, {sp.name}[{sp.index(e, f)}]);")
    out.append("  template <class Q>")
    out.append(
        "  static __device__ __forceinline__ void vrr(double* __restrict__ U, double* __restrict__ WA,"
        " double* __restrict__ WB, double* __restrict__ WC, const double* __restrict__ Fp, const Q& q,"
        " double a2, double b2, double c2) {"
    )
    out += ["    " + ln for ln in em.lines]
    out += ["    " + ln for ln in acc_lines]
    out.append("  }")
    # HRR: out[(3*centre + i) * NOUT + k]
    em2 = Emitter("h")
    hU, hA, hB, hC = HRR(em2, U), HRR(em2, WA), HRR(em2, WB), HRR(em2, WC)
    st = []
    k = 0
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    for i in range(3):
                        tA = hA.get(sh(a, i, 1), b, c, d)
                        if a[i] > 0:
                            tA = f"{tA} - {float(a[i])!r} * {hU.get(sh(a, i, -1), b, c, d)}"
                        tB = hB.get(a, sh(b, i, 1), c, d)
                        if b[i] > 0:
                            tB = f"{tB} - {float(b[i])!r} * {hU.get(a, sh(b, i, -1), c, d)}"
                        tC = hC.get(a, b, sh(c, i, 1), d)
                        if c[i] > 0:
                            tC = f"{tC} - {float(c[i])!r} * {hU.get(a, b, sh(c, i, -1), d)}"
                        st.append(f"out[{(0 + i) * nout + k}] = {tA};")
                        st.append(f"out[{(3 + i) * nout + k}] = {tB};")
                        st.append(f"out[{(6 + i) * nout + k}] = {tC};")
                    k += 1
    out.append(
        "  static __device__ __forceinline__ void hrr(const double* __restrict__ U, const double* __restrict__ WA,"
        " const double* __restrict__ WB, const double* __restrict__ WC, double* __restrict__ out,"
        " double ABx, double ABy, double ABz, double CDx, double CDy, double CDz) {"
    )
    out.append("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    out += ["    " + ln for ln in em2.lines]
    out += ["    " + ln for ln in st]
    out.append("  }")
    out.append("};")
    return "\n".join(out)


# ----------------------------------------------------------------------------------
# Table-driven programs for the warp-cooperative engine (large classes).
# ----------------------------------------------------------------------------------
# VRR node (uint4): x = dst | s1<<16, y = s2 | s3<<16, z = s4 | s5<<16,
#                   w = side | dir<<1 | k<<3 | ne<<8
#   V[dst] = c1[side,dir] V[s1] + c2[side,dir] V[s2] + k half[side] (V[s3] - ro[side] V[s4])
#            + ne oo2ze V[s5]
# slots 0..S hold pref*F_m, slot S+1 holds 0.
# HRR node (uint2): x = dst | s1<<16, y = s2 | side<<16 | dir<<17 ;  V[dst] = V[s1] + g[side,dir] V[s2]
# HRR leaves are the accumulators (slot = accumulator index).
COOP_CLASSES = {(2, 1, 2, 1), (2, 2, 1, 1), (2, 2, 2, 1), (2, 2, 2, 2)}


class VRRDag:
    def __init__(self, S):
        self.S = S
        self.ZERO = S + 1
        self.slot = {}
        self.nodes = []  # (dst, s1, s2, s3, s4, s5, side, dir, k, ne, level)
        self.level = {}

    def get(self, e, f, m):
        key = (e, f, m)
        if key in self.slot:
            return self.slot[key]
        if sum(e) == 0 and sum(f) == 0:
            return m
        Z = self.ZERO
        if sum(f) == 0:
            i = first_dir(e)
            n = e[i]
            s1 = self.get(sh(e, i, -1), f, m)
            s2 = self.get(sh(e, i, -1), f, m + 1)
            s3 = self.get(sh(e, i, -2), f, m) if n >= 2 else Z
            s4 = self.get(sh(e, i, -2), f, m + 1) if n >= 2 else Z
            ops = (s1, s2, s3, s4, Z)
            side, d, k, ne = 0, i, max(n - 1, 0), 0
        else:
            j = first_dir(f)
            nf = f[j]
            s1 = self.get(e, sh(f, j, -1), m)
            s2 = self.get(e, sh(f, j, -1), m + 1)
            s3 = self.get(e, sh(f, j, -2), m) if nf >= 2 else Z
            s4 = self.get(e, sh(f, j, -2), m + 1) if nf >= 2 else Z
            s5 = self.get(sh(e, j, -1), sh(f, j, -1), m + 1) if e[j] >= 1 else Z
            ops = (s1, s2, s3, s4, s5)
            side, d, k, ne = 1, j, max(nf - 1, 0), e[j]
        lvl = 1 + max(self.level.get(o, 0) for o in ops)
        dst = self.S + 2 + len(self.nodes)
        self.nodes.append((dst,) + ops + (side, d, k, ne, lvl))
        self.level[dst] = lvl
        self.slot[key] = dst
        return dst


class HRRDag:
    def __init__(self, acc):
        self.acc = acc
        self.slot = {}
        self.nodes = []  # (dst, s1, s2, side, dir, level)
        self.level = {}
        self.next = acc.size

    def get(self, a, b, c, d):
        key = (a, b, c, d)
        if key in self.slot:
            return self.slot[key]
        if sum(d) > 0:
            j = first_dir(d)
            s1 = self.get(a, b, sh(c, j, 1), sh(d, j, -1))
            s2 = self.get(a, b, c, sh(d, j, -1))
            side, dr = 1, j
        elif sum(b) > 0:
            i = first_dir(b)
            s1 = self.get(sh(a, i, 1), sh(b, i, -1), c, d)
            s2 = self.get(a, sh(b, i, -1), c, d)
            side, dr = 0, i
        else:
            r = self.acc.index(a, c)
            self.slot[key] = r
            return r
        lvl = 1 + max(self.level.get(s1, 0), self.level.get(s2, 0))
        dst = self.next
        self.next += 1
        self.nodes.append((dst, s1, s2, side, dr, lvl))
        self.level[dst] = lvl
        self.slot[key] = dst
        return dst


def _realloc(simple, nodes, pinned, nfixed, kind):
    """Reassign slots so a slot is reused once every reader sits in an earlier
    level (nodes of one level run concurrently).  Fixed slots [0, nfixed) hold
    the leaves; pinned slots are read after the last level."""
    last = {}
    for dst, ops, lvl in simple:
        for o in ops:
            last[o] = max(last.get(o, 0), lvl)
    INF = 1 << 30
    for p in pinned:
        last[p] = INF
    levels = sorted(set(l for _, _, l in simple))
    remap = {i: i for i in range(nfixed)}
    free = []
    nxt = nfixed
    by_level = {}
    for dst, ops, lvl in simple:
        by_level.setdefault(lvl, []).append(dst)
    released = set()
    for L in levels:
        # release slots whose readers all precede level L
        for old_slot, lu in list(last.items()):
            if lu < L and old_slot in remap and old_slot not in released:
                released.add(old_slot)
                free.append(remap[old_slot])
        for dst in by_level[L]:
            if free:
                remap[dst] = free.pop()
            else:
                remap[dst] = nxt
                nxt += 1
    out = []
    for n in nodes:
        if kind == "v":
            dst, s1, s2, s3, s4, s5 = n[:6]
            out.append((remap[dst], remap.get(s1, s1), remap.get(s2, s2), remap.get(s3, s3), remap.get(s4, s4),
                        remap.get(s5, s5)) + tuple(n[6:]))
        else:
            dst, s1, s2 = n[:3]
            out.append((remap[dst], remap.get(s1, s1), remap.get(s2, s2)) + tuple(n[3:]))
    return out, [remap.get(p, p) for p in pinned], max(nxt, nfixed)


def coop_program(la, lb, lc, ld):
    S = la + lb + lc + ld
    acc = AccSpace("acc", la, la + lb, lc, lc + ld)
    vd = VRRDag(S)
    targets = [vd.get(e, f, 0) for e, f in acc.targets()]
    vnodes = sorted(vd.nodes, key=lambda n: n[-1])
    vlev = []
    for lv in range(1, max((n[-1] for n in vnodes), default=0) + 1):
        vlev.append(sum(1 for n in vnodes if n[-1] < lv))
    vlev.append(len(vnodes))
    hd = HRRDag(acc)
    outs = []
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    outs.append(hd.get(a, b, c, d))
    hnodes = sorted(hd.nodes, key=lambda n: n[-1])
    hlev = []
    if hnodes:
        for lv in range(1, max(n[-1] for n in hnodes) + 1):
            hlev.append(sum(1 for n in hnodes if n[-1] < lv))
    hlev.append(len(hnodes))
    # liveness-based slot reuse (targets / outputs stay pinned to the end)
    vnodes, targets, vslots = _realloc([(n[0], n[1:6], n[-1]) for n in vnodes], vnodes, targets, S + 2, "v")
    hnodes, outs, hslots = _realloc([(n[0], n[1:3], n[-1]) for n in hnodes], hnodes, outs, acc.size, "h")
    return dict(S=S, vnodes=vnodes, vlev=vlev, targets=targets, hnodes=hnodes, hlev=hlev, outs=outs,
                vslots=vslots, hslots=hslots, nacc=acc.size)


def gen_coop(classes):
    lines = ["// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.",
             "// Programs of the warp-cooperative engine (large angular-momentum classes).",
             "#pragma once", "#include <stdint.h>", ""]
    vn, vl, tg, hn, hl, ou = [], [], [], [], [], []
    descs = []
    for cid, (la, lb, lc, ld) in classes:
        p = coop_program(la, lb, lc, ld)
        d = dict(cid=cid, la=la, lb=lb, lc=lc, ld=ld, S=p["S"], nacc=p["nacc"], nout=len(p["outs"]),
                 vslots=p["vslots"], hslots=p["hslots"], vnode_off=len(vn), nvlev=len(p["vlev"]) - 1,
                 vlev_off=len(vl), tgt_off=len(tg), hnode_off=len(hn), nhlev=len(p["hlev"]) - 1, hlev_off=len(hl),
                 out_off=len(ou))
        for (dst, s1, s2, s3, s4, s5, side, dr, k, ne, lvl) in p["vnodes"]:
            assert max(dst, s1, s2, s3, s4, s5) < 65536
            vn.append((dst | s1 << 16, s2 | s3 << 16, s4 | s5 << 16, side | dr << 1 | k << 3 | ne << 8))
        vl += p["vlev"]
        tg += p["targets"]
        for (dst, s1, s2, side, dr, lvl) in p["hnodes"]:
            assert max(dst, s1, s2) < 65536
            hn.append((dst | s1 << 16, s2 | side << 16 | dr << 17))
        hl += p["hlev"]
        ou += p["outs"]
        descs.append(d)
    fields = ["cid", "la", "lb", "lc", "ld", "S", "nacc", "nout", "vslots", "hslots", "vnode_off", "nvlev", "vlev_off",
              "tgt_off", "hnode_off", "nhlev", "hlev_off", "out_off"]
    lines.append("struct CoopClass { int " + ", ".join(fields) + "; };")
    lines.append(f"#define QX_NUM_COOP {len(descs)}")
    lines.append("static const CoopClass g_coop_classes[QX_NUM_COOP] = {")
    for d in descs:
        lines.append("  {" + ", ".join(str(d[f]) for f in fields) + "},")
    lines.append("};")
    def arr(name, typ, vals, per):
        out = [f"__device__ const {typ} {name}[{max(len(vals), 1)}] = {{"]
        row = []
        for v in vals:
            row.append(per(v))
            if len(row) == 8:
                out.append("  " + ", ".join(row) + ",")
                row = []
        if row:
            out.append("  " + ", ".join(row) + ",")
        if not vals:
            out.append("  {}" if typ.startswith("uint") else "  0")
        out.append("};")
        return out
    lines += arr("g_coop_vnodes", "uint4", vn, lambda v: "{%du,%du,%du,%du}" % v)
    lines += arr("g_coop_vlev", "int", vl, str)
    lines += arr("g_coop_targets", "unsigned short", tg, str)
    lines += arr("g_coop_hnodes", "uint2", hn, lambda v: "{%du,%du}" % v)
    lines += arr("g_coop_hlev", "int", hl, str)
    lines += arr("g_coop_outs", "unsigned short", ou, str)
    return "\n".join(lines) + "\n"


# ----------------------------------------------------------------------------------
# First-derivative programs (cooperative engine).  Accumulator sets, in order:
#   U  = sum [e0|f0]          e in [la-1, lab],   f in [lc-1, lcd]
#   WA = sum 2 alpha [e0|f0]  e in [la+1, lab+1], f in [lc, lcd]
#   WB = sum 2 beta  [e0|f0]  e in [la, lab+1],   f in [lc, lcd]
#   WC = sum 2 gamma [e0|f0]  e in [la, lab],     f in [lc+1, lcd+1]
# HRR outputs: 9 blocks (A_x,A_y,A_z,B_x,..,C_z) of n1*n2*n3*n4 each:
#   dA_i = (a+1_i b|cd)_WA - a_i (a-1_i b|cd)_U   (likewise B on b, C on c);
# combination nodes use g = -k (geometry slots 6.. hold -1, -2, -3, -4).
# ----------------------------------------------------------------------------------
class HRRMulti:
    def __init__(self, spaces):
        self.spaces = spaces  # name -> (AccSpace, offset)
        self.slot = {}
        self.nodes = []
        self.level = {}
        self.next = sum(sp.size for sp, _ in spaces.values())

    def _new(self, s1, s2, side, dr):
        lvl = 1 + max(self.level.get(s1, 0), self.level.get(s2, 0))
        dst = self.next
        self.next += 1
        self.nodes.append((dst, s1, s2, side, dr, lvl))
        self.level[dst] = lvl
        return dst

    def get(self, sp, a, b, c, d):
        key = (sp, a, b, c, d)
        if key in self.slot:
            return self.slot[key]
        if sum(d) > 0:
            j = first_dir(d)
            dst = self._new(self.get(sp, a, b, sh(c, j, 1), sh(d, j, -1)), self.get(sp, a, b, c, sh(d, j, -1)), 1, j)
        elif sum(b) > 0:
            i = first_dir(b)
            dst = self._new(self.get(sp, sh(a, i, 1), sh(b, i, -1), c, d), self.get(sp, a, sh(b, i, -1), c, d), 0, i)
        else:
            lm = getattr(self, "leafmap", None)
            if lm is not None:
                dst = lm[(sp, a, c)]
            else:
                acc, off = self.spaces[sp]
                dst = off + acc.index(a, c)
        self.slot[key] = dst
        return dst

    def combine(self, x, y, k):
        """x - k*y (k = 1..4)"""
        return self._new(x, y, 2, k - 1)


def coop_deriv_program(la, lb, lc, ld):
    lab, lcd = la + lb, lc + ld
    S = lab + lcd + 1
    spaces = [("U", AccSpace("U", la - 1, lab, lc - 1, lcd)), ("WA", AccSpace("WA", la + 1, lab + 1, lc, lcd)),
              ("WB", AccSpace("WB", la, lab + 1, lc, lcd)), ("WC", AccSpace("WC", la, lab, lc + 1, lcd + 1))]
    vd = VRRDag(S)
    targets = []
    sizes = []
    for name, sp in spaces:
        sizes.append(sp.size)
        targets += [vd.get(e, f, 0) for e, f in sp.targets()]
    vnodes = sorted(vd.nodes, key=lambda n: n[-1])
    vlev = [sum(1 for n in vnodes if n[-1] < lv) for lv in range(1, max(n[-1] for n in vnodes) + 1)] + [len(vnodes)]
    offs = {}
    o = 0
    for name, sp in spaces:
        offs[name] = (sp, o)
        o += sp.size
    hm = HRRMulti(offs)
    outs = [None] * (9 * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld))
    nout = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    k = 0
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    for i in range(3):
                        x = hm.get("WA", sh(a, i, 1), b, c, d)
                        outs[(0 + i) * nout + k] = hm.combine(x, hm.get("U", sh(a, i, -1), b, c, d), a[i]) if a[i] else x
                        x = hm.get("WB", a, sh(b, i, 1), c, d)
                        outs[(3 + i) * nout + k] = hm.combine(x, hm.get("U", a, sh(b, i, -1), c, d), b[i]) if b[i] else x
                        x = hm.get("WC", a, b, sh(c, i, 1), d)
                        outs[(6 + i) * nout + k] = hm.combine(x, hm.get("U", a, b, sh(c, i, -1), d), c[i]) if c[i] else x
                    k += 1
    nacc = sum(sizes)
    # every output must be its own HRR node: the epilogue runs inline when the
    # node is evaluated, so outputs are not kept to the end
    # (an output that is a leaf, or a node another output already owns, gets an
    # identity node V[sl] + 0 * V[sl])
    owner = {}
    for ob, sl in enumerate(outs):
        if sl < nacc or sl in owner:
            sl = hm._new(sl, sl, 3, 0)
            outs[ob] = sl
        owner[sl] = ob
    hnodes = sorted(hm.nodes, key=lambda n: n[-1])
    hout = [owner.get(n[0], 0xFFFF) for n in hnodes]
    hlev = [sum(1 for n in hnodes if n[-1] < lv) for lv in range(1, max(n[-1] for n in hnodes) + 1)]
    hlev.append(len(hnodes))
    vnodes, targets, vslots = _realloc([(n[0], n[1:6], n[-1]) for n in vnodes], vnodes, targets, S + 2, "v")
    hnodes, _, hslots = _realloc([(n[0], n[1:3], n[-1]) for n in hnodes], hnodes, [], nacc, "h")
    return dict(S=S, vnodes=vnodes, vlev=vlev, targets=targets, hnodes=hnodes, hlev=hlev, hout=hout, vslots=vslots,
                hslots=hslots, nacc=nacc, sizes=sizes, nout=nout)


def gen_coop_deriv(classes):
    lines = ["// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.",
             "// First-derivative programs of the cooperative engine.", "#pragma once", "#include <stdint.h>", ""]
    vn, vl, tg, hn, hl, ou = [], [], [], [], [], []
    descs = []
    for cid, (la, lb, lc, ld) in classes:
        p = coop_deriv_program(la, lb, lc, ld)
        assert len(p["hout"]) == len(p["hnodes"])
        d = dict(cid=cid, la=la, lb=lb, lc=lc, ld=ld, S=p["S"], nacc=p["nacc"], nu=p["sizes"][0], na=p["sizes"][1],
                 nb=p["sizes"][2], nc=p["sizes"][3], nout=p["nout"], vslots=p["vslots"], hslots=p["hslots"],
                 vnode_off=len(vn), nvlev=len(p["vlev"]) - 1, vlev_off=len(vl), tgt_off=len(tg), hnode_off=len(hn),
                 nhlev=len(p["hlev"]) - 1, hlev_off=len(hl), out_off=len(ou))
        for (dst, s1, s2, s3, s4, s5, side, dr, k, ne, lvl) in p["vnodes"]:
            assert max(dst, s1, s2, s3, s4, s5) < 65536
            vn.append((dst | s1 << 16, s2 | s3 << 16, s4 | s5 << 16, side | dr << 1 | k << 3 | ne << 8))
        vl += p["vlev"]
        tg += p["targets"]
        for (dst, s1, s2, side, dr, lvl) in p["hnodes"]:
            assert max(dst, s1, s2) < 65536
            hn.append((dst | s1 << 16, s2 | side << 16 | dr << 18))
        hl += p["hlev"]
        ou += p["hout"]
        descs.append(d)
    fields = ["cid", "la", "lb", "lc", "ld", "S", "nacc", "nu", "na", "nb", "nc", "nout", "vslots", "hslots",
              "vnode_off", "nvlev", "vlev_off", "tgt_off", "hnode_off", "nhlev", "hlev_off", "out_off"]
    lines.append("struct DerClass { int " + ", ".join(fields) + "; };")
    lines.append(f"#define QX_NUM_DER {len(descs)}")
    lines.append("static const DerClass g_der_classes[QX_NUM_DER] = {")
    for d in descs:
        lines.append("  {" + ", ".join(str(d[f]) for f in fields) + "},")
    lines.append("};")

    def arr(name, typ, vals, per):
        out = [f"__device__ const {typ} {name}[{max(len(vals), 1)}] = {{"]
        for i0 in range(0, len(vals), 8):
            out.append("  " + ", ".join(per(v) for v in vals[i0:i0 + 8]) + ",")
        out.append("};")
        return out
    lines += arr("g_der_vnodes", "uint4", vn, lambda v: "{%du,%du,%du,%du}" % v)
    lines += arr("g_der_vlev", "int", vl, str)
    lines += arr("g_der_targets", "unsigned short", tg, str)
    lines += arr("g_der_hnodes", "uint2", hn, lambda v: "{%du,%du}" % v)
    lines += arr("g_der_hlev", "int", hl, str)
    lines += arr("g_der_outs", "unsigned short", ou, str)
    return "\n".join(lines) + "\n"


# ----------------------------------------------------------------------------------
# Algorithmic FLOP counts (the roofline's work unit).  Counting rule, fixed:
#   VRR node: c1*x + c2*y = 3; the e_i/(2 zeta) term +4; the coupling term +2;
#   target accumulation 1 (plain) / 2 (weighted derivative sets);
#   primitive set-up (P-Q geometry, Boys Taylor + downward recursion, exp) 60;
#   HRR node 2 per contracted quartet (identity copies 0).
# ----------------------------------------------------------------------------------
SETUP_FLOPS = 60


def vrr_node_flops(k, ne):
    return 3 + (4 if k else 0) + (2 if ne else 0)


def class_flops(la, lb, lc, ld):
    p = coop_program(la, lb, lc, ld)
    vrr = SETUP_FLOPS + sum(vrr_node_flops(n[8], n[9]) for n in p["vnodes"]) + len(p["targets"])
    hrr = 2 * len(p["hnodes"])
    d = coop_deriv_program(la, lb, lc, ld)
    dvrr = SETUP_FLOPS + sum(vrr_node_flops(n[8], n[9]) for n in d["vnodes"]) + 2 * len(d["targets"])
    dhrr = 2 * sum(1 for n in d["hnodes"] if n[3] != 3)
    return vrr, hrr, dvrr, dhrr


# ----------------------------------------------------------------------------------
# Warp-per-quartet kernels (qx_warp.cuh): lanes = primitive quartets.  The class's
# straight-line VRR runs in each lane; its targets become "items" in emission
# order (derivative targets once per accumulator set, times the set weight), which
# are staged 16 at a time and folded across the warp by reduce16 into the warp's
# shared accumulators.  The HRR tables are built over that item order.
# ----------------------------------------------------------------------------------
WARP_PEAK_MAX = 400  # VRR values a lane may keep live (registers, spills to L1 beyond)


def _warp_targets(la, lb, lc, ld, deriv):
    lab, lcd = la + lb, lc + ld
    if not deriv:
        acc = AccSpace("acc", la, lab, lc, lcd)
        return [((e, f), ["acc"]) for e, f in reversed(list(acc.targets()))], {"acc": acc}
    if deriv == 2:
        spaces = {"U": AccSpace("U", la - 2, lab, lc - 2, lcd), "WA": AccSpace("WA", la, lab + 1, lc - 1, lcd),
                  "WB": AccSpace("WB", la - 1, lab + 1, lc - 1, lcd), "WC": AccSpace("WC", la - 1, lab, lc, lcd + 1),
                  "AA": AccSpace("AA", la + 2, lab + 2, lc, lcd), "BB": AccSpace("BB", la, lab + 2, lc, lcd),
                  "CC": AccSpace("CC", la, lab, lc + 2, lcd + 2), "AB": AccSpace("AB", la + 1, lab + 2, lc, lcd),
                  "AC": AccSpace("AC", la + 1, lab + 1, lc + 1, lcd + 1),
                  "BC": AccSpace("BC", la, lab + 1, lc + 1, lcd + 1)}
    else:
        spaces = {"U": AccSpace("U", la - 1, lab, lc - 1, lcd), "WA": AccSpace("WA", la + 1, lab + 1, lc, lcd),
                  "WB": AccSpace("WB", la, lab + 1, lc, lcd), "WC": AccSpace("WC", la, lab, lc + 1, lcd + 1)}
    member = {}
    for name in spaces:
        for t in spaces[name].targets():
            member.setdefault(t, []).append(name)
    order = sorted(member, key=lambda t: (-sum(t[0]), -sum(t[1]), gidx(t[0]), gidx(t[1])))
    return [(t, member[t]) for t in order], spaces


def _peak_live(lines, consumed_at):
    """Peak live count of SSA values in `lines` (values die at their last use)."""
    import re as _re
    uses = {}
    defs = []
    for i, ln in enumerate(lines):
        m = _re.match(r"const \w+ (v\d+(?:_\d+)?) = (.*);", ln)
        body = m.group(2) if m else ln
        for d in _re.findall(r"\b(v\d+(?:_\d+)?)\b", body):
            uses[d] = i
        defs.append(m.group(1) if m else None)
    alive, pk = set(), 0
    for i, ln in enumerate(lines):
        if defs[i]:
            alive.add(defs[i])
            pk = max(pk, len(alive))
        for d in list(alive):
            if uses.get(d, -1) <= i and d != defs[i]:
                alive.discard(d)
    return pk


# Live VRR values (doubles, two registers each) one chunk of a derivative
# program may keep.  Straight-line code above that spills to local memory; below
# it the program is cut into chunks that each recompute the intermediates they
# need from the saved inputs (see qx_load_inputs), so no chunk's values outlive it.
WARP_LIVE_BUDGET = {0: None, 1: 80, 2: None}

_TARGET_ORDERS = {
    # highest bra AM first (the order of the plain programs)
    "bra_desc": lambda t: (-sum(t[0]), -sum(t[1]), gidx(t[0]), gidx(t[1])),
    # lowest bra AM first: fewer live values per chunk for the derivative programs
    "bra_asc": lambda t: (sum(t[0]), gidx(t[0]), sum(t[1]), gidx(t[1])),
}


def _chunk_cost(tl):
    """(FP ops, peak live values) of the straight-line VRR for the targets tl."""
    em = Emitter("v")
    vr = VRR(em)
    for (e, f), sets in tl:
        v = vr.get(e, f, 0)
        for _ in sets:
            em.lines.append(f"stg[0] = {v};")
    ops = sum(ln.count("*") + ln.count(" + ") + ln.count(" - ") for ln in em.lines if ln.startswith("const"))
    return ops, _peak_live(em.lines, None)


def _chunks(tl, budget):
    """Greedy cut of tl into contiguous chunks whose peak live count fits the budget."""
    out, s = [], 0
    while s < len(tl):
        lo, hi = s + 1, len(tl)
        while lo < hi:
            mid = (lo + hi + 1) // 2
            if _chunk_cost(tl[s:mid])[1] <= budget:
                lo = mid
            else:
                hi = mid - 1
        out.append((s, lo))
        s = lo
    return out


def _plan_targets(tlist, budget):
    """Target order and chunk bounds: one chunk if it fits, else the order with the
    fewest recomputed operations."""
    if budget is None or _chunk_cost(tlist)[1] <= budget:
        return tlist, [(0, len(tlist))]
    best = None
    for key in _TARGET_ORDERS.values():
        tl = sorted(tlist, key=lambda x: key(x[0]))
        ch = _chunks(tl, budget)
        ops = sum(_chunk_cost(tl[a:b])[0] for a, b in ch)
        if best is None or ops < best[0]:
            best = (ops, tl, ch)
    return best[1], best[2]


def warp_program(la, lb, lc, ld, deriv):
    import re as _re
    S = la + lb + lc + ld + deriv
    tlist, spaces = _warp_targets(la, lb, lc, ld, deriv)
    tlist, chunks = _plan_targets(tlist, WARP_LIVE_BUDGET[deriv])
    items = []  # (space, e, f)
    leaf = {}
    wname = {"acc": None, "U": None, "WA": "wa", "WB": "wb", "WC": "wc", "AA": "wa * wa", "BB": "wb * wb",
             "CC": "wc * wc", "AB": "wa * wb", "AC": "wa * wc", "BC": "wb * wc"}
    lines = []
    peak = 0
    for ci, (c0, c1) in enumerate(chunks):
        em = Emitter(f"v{ci}_" if len(chunks) > 1 else "v", "T")
        vr = VRR(em)
        for (e, f), sets in tlist[c0:c1]:
            v = vr.get(e, f, 0)
            for sp in sets:
                k = len(items)
                items.append((sp, e, f))
                leaf[(sp, e, f)] = k
                w = wname[sp]
                # items are staged and summed in FP64 whatever the recurrence type
                em.lines.append(f"stg[{k % 16}] = (double){v};" if w is None
                                else f"stg[{k % 16}] = {w} * (double){v};")
                if k % 16 == 15:
                    em.lines.append(f"sink(stg, {k - 15}, lane);")
        peak = max(peak, _peak_live(em.lines, None))
        if ci == 0:
            if len(chunks) > 1:
                lines.append(f"qx_save_inputs<{S + 1}>(q, Fp, save, lane);")
            lines += em.lines
        else:
            # the inputs again, by volatile loads of the lane's saved copy: the
            # compiler cannot merge this chunk's intermediates with an earlier
            # chunk's, whose values are dead by now
            lines.append("{")
            lines.append(f"  T Fc[{S + 1}];")
            lines.append("  PrimQT<T> qc;")
            lines.append(f"  qx_load_inputs<{S + 1}>(save, lane, qc, Fc);")
            for ln in em.lines:
                ln = ln.replace("Fp[", "Fc[")
                lines.append("  " + _re.sub(r"\bq\.", "qc.", ln))
            lines.append("}")
    em = Emitter("v")
    em.lines = lines
    nitem = len(items)
    if nitem % 16:
        for k in range(nitem, (nitem + 15) // 16 * 16):
            em.lines.append(f"stg[{k % 16}] = 0.0;")
        em.lines.append(f"sink(stg, {(nitem // 16) * 16}, lane);")
    nitem_pad = (nitem + 15) // 16 * 16
    # HRR over the item layout
    nout = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    if not deriv:
        hm = HRRMulti({"acc": (spaces["acc"], 0)})
        hm.next = nitem_pad
        hm.leafmap = leaf
        outs = [hm.get("acc", a, b, c, d) for a in comps(la) for b in comps(lb) for c in comps(lc) for d in comps(ld)]
        hnodes = sorted(hm.nodes, key=lambda n: n[-1])
        hout = None
        pinned = outs
    elif deriv == 2:
        hm = HRRMulti({k: (v, 0) for k, v in spaces.items()})
        hm.next = nitem_pad
        hm.leafmap = leaf
        pairs = [(P, Q) for P in range(9) for Q in range(P, 9)]
        outs = [None] * (len(pairs) * nout)
        setname = {(): "U", (0,): "WA", (1,): "WB", (2,): "WC", (0, 0): "AA", (1, 1): "BB", (2, 2): "CC",
                   (0, 1): "AB", (0, 2): "AC", (1, 2): "BC"}
        kk = 0
        for a in comps(la):
            for b in comps(lb):
                for c in comps(lc):
                    for d in comps(ld):
                        for pi, (P, Q) in enumerate(pairs):
                            X, i = divmod(P, 3)
                            Y, j = divmod(Q, 3)
                            terms = []
                            for fx in (0, 1):
                                for fy in (0, 1):
                                    cm = [list(a), list(b), list(c), list(d)]
                                    coef = 1
                                    if fx == 0:
                                        cm[X][i] += 1
                                    else:
                                        coef *= -cm[X][i]
                                        cm[X][i] -= 1
                                    if coef == 0:
                                        continue
                                    if fy == 0:
                                        cm[Y][j] += 1
                                    else:
                                        coef *= -cm[Y][j]
                                        cm[Y][j] -= 1
                                    if coef == 0 or min(min(t) for t in cm) < 0:
                                        continue
                                    wset = tuple(sorted(([X] if fx == 0 else []) + ([Y] if fy == 0 else [])))
                                    terms.append((hm.get(setname[wset], *[tuple(t) for t in cm]), coef))
                            # merge equal slots, then chain x + c y nodes (constants in -8..7)
                            merged = {}
                            for sl, cf in terms:
                                merged[sl] = merged.get(sl, 0) + cf
                            terms = [(sl, cf) for sl, cf in merged.items() if cf != 0]
                            if not terms:
                                raise RuntimeError("second-derivative output with no terms")
                            sl0, c0 = terms[0]
                            node = sl0 if c0 == 1 else hm._new(sl0, sl0, 4, c0 - 1)
                            for sl, cf in terms[1:]:
                                node = hm._new(node, sl, 4, cf)
                            outs[pi * nout + kk] = node
                        kk += 1
        owner = {}
        for ob, sl in enumerate(outs):
            if sl < nitem_pad or sl in owner:
                sl = hm._new(sl, sl, 3, 0)
                outs[ob] = sl
            owner[sl] = ob
        hnodes = sorted(hm.nodes, key=lambda n: n[-1])
        hout = [owner.get(n[0], 0xFFFF) for n in hnodes]
        pinned = []
    else:
        hm = HRRMulti({k: (v, 0) for k, v in spaces.items()})
        hm.next = nitem_pad
        hm.leafmap = leaf
        outs = [None] * (9 * nout)
        kk = 0
        for a in comps(la):
            for b in comps(lb):
                for c in comps(lc):
                    for d in comps(ld):
                        for i in range(3):
                            x = hm.get("WA", sh(a, i, 1), b, c, d)
                            outs[i * nout + kk] = hm.combine(x, hm.get("U", sh(a, i, -1), b, c, d), a[i]) if a[i] else x
                            x = hm.get("WB", a, sh(b, i, 1), c, d)
                            outs[(3 + i) * nout + kk] = hm.combine(x, hm.get("U", a, sh(b, i, -1), c, d), b[i]) if b[i] else x
                            x = hm.get("WC", a, b, sh(c, i, 1), d)
                            outs[(6 + i) * nout + kk] = hm.combine(x, hm.get("U", a, b, sh(c, i, -1), d), c[i]) if c[i] else x
                        kk += 1
        owner = {}
        for ob, sl in enumerate(outs):
            if sl < nitem_pad or sl in owner:
                sl = hm._new(sl, sl, 3, 0)
                outs[ob] = sl
            owner[sl] = ob
        hnodes = sorted(hm.nodes, key=lambda n: n[-1])
        hout = [owner.get(n[0], 0xFFFF) for n in hnodes]
        pinned = []
    hlev = [sum(1 for n in hnodes if n[-1] < lv) for lv in range(1, max((n[-1] for n in hnodes), default=0) + 1)]
    hlev.append(len(hnodes))
    hnodes2, pinned2, hslots = _realloc([(n[0], n[1:3], n[-1]) for n in hnodes], hnodes, pinned, nitem_pad, "h")
    vmap = None
    if deriv == 1:
        # item -> accumulator index of the cooperative derivative layout (spaces
        # U, WA, WB, WC back to back), for the global-accumulator VRR kernel
        offs, o = {}, 0
        for name in ("U", "WA", "WB", "WC"):
            offs[name] = o
            o += spaces[name].size
        vmap = [offs[sp] + spaces[sp].index(e, f) for sp, e, f in items] + [0xFFFF] * (nitem_pad - nitem)
    return dict(S=S, lines=em.lines, nitem=nitem, nitem_pad=nitem_pad, peak=peak, hnodes=hnodes2, hlev=hlev,
                outs=pinned2 if not deriv else hout, hslots=max(hslots, nitem_pad), nout=nout, vmap=vmap,
                nchunk=len(chunks))


def warp_feasible(la, lb, lc, ld, deriv):
    p = warp_program(la, lb, lc, ld, deriv)
    return p["peak"] <= WARP_PEAK_MAX and warp_smem(p, deriv) <= WARP_SMEM_MAX, p


def wvrr_wanted(la, lb, lc, ld):
    """Classes that also get the global-accumulator derivative VRR kernel: the ones
    with long primitive loops and large accumulator sets."""
    return la + lb + lc + ld >= 4


def pvrr_wanted(la, lb, lc, ld):
    """Classes that also get the global-accumulator plain VRR kernel (split mode)."""
    return la + lb + lc + ld >= 6


WARP_SMEM_MAX = (227 * 1024) // (8 * 4)  # doubles of shared memory per warp (4 warps per block)


def warp_save(p):
    """Per-warp input save area (doubles) of a chunked program: 17 PrimQ scalars and
    S + 1 Boys values per lane."""
    return (17 + p["S"] + 1) * 32 if p["nchunk"] > 1 else 0


def warp_smem(p, deriv):
    return p["hslots"] + 32 + (p["nout"] if deriv in (1, 2) else 0) + warp_save(p)


def gen_warp_code(cid, la, lb, lc, ld, deriv, p, want_warp=True, want_wvrr=False):
    """Warp program of one class: the k_warp kernel (accumulators in shared memory,
    HRR and epilogue in the same kernel) and/or, for first derivatives, the
    global-accumulator VRR kernel k_wvrr that feeds the cooperative HRR pass."""
    tag = f"{'pdh'[deriv]}{cid:02d}"
    L = []
    def gidx(side, dr):
        # geometry / constant slot of the kernel's table: AB 0..2, CD 3..5, 6 + (c + 8) for a constant c
        if side == 0:
            return dr
        if side == 1:
            return 3 + dr
        c = -(dr + 1) if side == 2 else (0 if side == 3 else dr)
        assert -8 <= c <= 7, c
        return 6 + c + 8
    def arr(name, typ, vals, per):
        out = [f"static __device__ const {typ} {name}[{max(len(vals), 1)}] = {{"]
        for i0 in range(0, len(vals), 8):
            out.append("  " + ", ".join(per(v) for v in vals[i0:i0 + 8]) + ",")
        if not vals:
            out.append("  {}" if typ.startswith("uint") else "  0")
        out.append("};")
        return out
    if want_warp:
        hn = [(dst | s1 << 16, s2 | gidx(side, dr) << 16) for (dst, s1, s2, side, dr, lvl) in p["hnodes"]]
        for n in hn:
            assert n[0] < 2**32
        L += arr(f"k_hn_{tag}", "uint2", hn, lambda v: "{%du,%du}" % v)
        L += arr(f"k_hl_{tag}", "int", p["hlev"], str)
        L += arr(f"k_ho_{tag}", "unsigned short", p["outs"], str)
    if want_wvrr and deriv:
        assert p["vmap"] is not None and max(p["vmap"]) <= 0xFFFF
        L += arr(f"k_vm_{tag}", "unsigned short", p["vmap"], str)
    L.append(f"struct Warp_{tag} {{")
    L.append(f"  static constexpr int LA = {la}, LB = {lb}, LC = {lc}, LD = {ld};")
    L.append(f"  static constexpr int S = {p['S']}, NITEM = {p['nitem']}, NITEM_PAD = {p['nitem_pad']};")
    L.append(f"  static constexpr int HSLOTS = {p['hslots']}, NOUT = {p['nout']}, NHLEV = {len(p['hlev']) - 1};")
    L.append(f"  static constexpr int SMEM_PER_WARP = {warp_smem(p, deriv)};")
    L.append(f"  static constexpr int NCHUNK = {p['nchunk']};  // VRR chunks (recomputed intermediates)")
    L.append(f"  static constexpr int SAVE = {warp_save(p)};  // per-warp input save area (doubles)")
    if want_warp:
        L.append(f"  static __device__ __forceinline__ const uint2* hnodes() {{ return k_hn_{tag}; }}")
        L.append(f"  static __device__ __forceinline__ const int* hlev() {{ return k_hl_{tag}; }}")
        L.append(f"  static __device__ __forceinline__ const unsigned short* outs() {{ return k_ho_{tag}; }}")
    if want_wvrr and deriv:
        L.append(f"  static __device__ __forceinline__ const unsigned short* vmap() {{ return k_vm_{tag}; }}")
    L.append("  // T = double, or float for the mixed-precision quartets (staging stays FP64)")
    L.append("  template <class T, class Sink>")
    L.append("  static __device__ __forceinline__ void vrr(const T* __restrict__ Fp, const PrimQT<T>& q, double wa,"
             " double wb, double wc, const Sink& sink, unsigned lane, T* save) {")
    L.append("    (void)wa; (void)wb; (void)wc; (void)save;")
    L.append("    double stg[16];")
    L += ["    " + ln for ln in p["lines"]]
    L.append("  }")
    L.append("};")
    if want_warp:
        L.append(f"void qx_launch_warp_{tag}(const qx::WarpArgs& w, int mode, cudaStream_t s) "
                 f"{{ qx::launch_warp<Warp_{tag}, {deriv}>(w, mode, s); }}")
    if want_wvrr:
        kind = "wvrr" if deriv else "pvrr"
        L.append(f"void qx_launch_{kind}_{tag}(const qx::EriArgs& a, const int2* tasks, long long ntask, int chunk, "
                 f"double* acc, int nacc, cudaStream_t s) "
                 f"{{ qx::launch_gvrr<Warp_{tag}, {'true' if deriv else 'false'}>(a, tasks, ntask, chunk, acc, nacc, s); }}")
    if want_wvrr and want_warp and deriv == 1:
        # derivative split with the warp HRR: items kept in item order
        L.append(f"void qx_launch_dsplit_{tag}(const qx::EriArgs& a, const int2* tasks, long long ntask, int chunk, "
                 f"double* acc, int nacc, cudaStream_t s) "
                 f"{{ qx::launch_gvrr<Warp_{tag}, true, true>(a, tasks, ntask, chunk, acc, nacc, s); }}")
    return "\n".join(L)


def pair_classes(lmax):
    return [(a, b) for a in range(lmax + 1) for b in range(a + 1)]


def quartet_classes(lmax):
    pc = pair_classes(lmax)
    out = []
    for i, (la, lb) in enumerate(pc):
        for j, (lc, ld) in enumerate(pc[: i + 1]):
            out.append((la, lb, lc, ld))
    return out


class _Out:
    """File writer that leaves an existing file untouched when its content is
    unchanged, so a regeneration does not force the (slow) recompilation of
    every generated translation unit."""

    def __init__(self, path, mode="w"):
        self.path, self.parts = path, []

    def __enter__(self):
        return self

    def write(self, text):
        self.parts.append(text)

    def __exit__(self, *exc):
        text = "".join(self.parts)
        if os.path.exists(self.path):
            with open(self.path) as f:
                if f.read() == text:
                    return
        with open(self.path, "w") as f:
            f.write(text)


# Highest shell angular momentum of the Rys engine (every class up to (ff|ff)).
RYS_LMAX = 3
RYS_ALL_KINDS = ("RK_PLAIN", "RK_GRAD", "RK_GRADL", "RK_HVP", "RK_GRADT", "RK_DER1", "RK_DER2", "RK_DER3",
                 "RK_DER4")


def gen_rys(here, lmax_os):
    """One translation unit per class up to RYS_LMAX with the Rys launcher
    qx_launch_rys_<id>(args, kind, mode, nwork, stream) -> 0, or 1 when the kind
    does not fit shared memory for the class.  Every class gets every kind: for
    the f classes this is the only engine, for the l <= lmax_os classes it
    serves the second- and higher-order derivatives and is an autotuner
    candidate next to the Obara-Saika programs."""
    del lmax_os
    qc = quartet_classes(RYS_LMAX)
    for i, (a, b, c, d) in enumerate(qc):
        kinds = RYS_ALL_KINDS
        L = ["// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.",
             f"// Rys-engine launchers of class ({a}{b}|{c}{d}).",
             '#include "../qx_rys.cuh"',
             f"int qx_launch_rys_{i:02d}(const qx::RysArgs& ra, int kind, int mode, long long nwork, cudaStream_t s) {{",
             "    switch (kind) {"]
        for k in kinds:
            L.append(f"    case qx::{k}: return qx::launch_rys<{a}, {b}, {c}, {d}, qx::{k}>(ra, mode, nwork, s) ? 0 : 1;")
        L += ["    default: return 1;", "    }", "}"]
        with _Out(os.path.join(here, "gen", f"k_rys_{i:02d}.cu")) as f:
            f.write("\n".join(L) + "\n")
    H = ["// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.", "#pragma once",
         f"#define QX_RYS_LMAX {RYS_LMAX}",
         f"#define QX_NCLS_ALL {len(qc)}",
         f"#define QX_NPCLS_ALL {len(pair_classes(RYS_LMAX))}",
         "// X(class_id, LA, LB, LC, LD) for every canonical class up to QX_RYS_LMAX",
         "#define QX_FOR_EACH_CLASS_ALL(X) " + " ".join(f"X({i:02d}, {a}, {b}, {c}, {d})" for i, (a, b, c, d) in enumerate(qc))]
    with _Out(os.path.join(here, "gen", "rys_index.cuh")) as f:
        f.write("\n".join(H) + "\n")


def main():
    lmax = int(sys.argv[1]) if len(sys.argv) > 1 else 2
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "gen"), exist_ok=True)
    hdr = [
        "// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.",
        "// QX_CLASS_*_FLOPS: VRR per primitive quartet, HRR per contracted quartet",
        "// (plain and first-derivative programs; counting rule in gen_eri.py).",
        f"// Canonical classes up to l = {lmax}.",
        "#pragma once",
        f"#define QX_GEN_LMAX {lmax}",
        "template <int LA, int LB, int LC, int LD> struct EriCls;",
        "template <int LA, int LB, int LC, int LD> struct DerCls;",
    ]
    qc = quartet_classes(lmax)
    hdr.append("// X(class_id, LA, LB, LC, LD) for every canonical quartet class")
    hdr.append("#define QX_FOR_EACH_CLASS(X) " + " ".join(f"X({i}, {a}, {b}, {c}, {d})" for i, (a, b, c, d) in enumerate(qc)))
    hdr.append(f"#define QX_NUM_CLASSES {len(qc)}")
    hdr.append(f"#define QX_NUM_PAIR_CLASSES {len(pair_classes(lmax))}")
    hdr.append("#define QX_CLASS_NOUT " + "{" + ", ".join(str(ncart(a) * ncart(b) * ncart(c) * ncart(d)) for (a, b, c, d) in qc) + "}")
    hdr.append("#define QX_CLASS_COOP " + "{" + ", ".join("1" if c in COOP_CLASSES else "0" for c in qc) + "}")
    hdr.append("#define QX_CLASS_NACC {" + ", ".join(str(AccSpace("a", a, a + b, c, c + d).size) for (a, b, c, d) in qc) + "}")
    hdr.append("// X(class_id, LA, LB, LC, LD) for the classes with straight-line kernels")
    hdr.append("#define QX_FOR_EACH_SL_CLASS(X) " + " ".join(f"X({i}, {a}, {b}, {c}, {d})" for i, (a, b, c, d) in enumerate(qc) if (a, b, c, d) not in COOP_CLASSES))
    fl = [class_flops(*c) for c in qc]
    for k, name in enumerate(("VRR", "HRR", "DVRR", "DHRR")):
        hdr.append(f"#define QX_CLASS_{name}_FLOPS " + "{" + ", ".join(str(f[k]) for f in fl) + "}")
    body = [gen_plain(*c) for c in qc if c not in COOP_CLASSES]
    with _Out(os.path.join(here, "gen", "coop_tables.cuh")) as f:
        f.write(gen_coop([(i, c) for i, c in enumerate(qc) if c in COOP_CLASSES]))
    with _Out(os.path.join(here, "gen", "eri_classes.cuh")) as f:
        f.write("\n".join(hdr) + "\n\n" + "\n\n".join(body) + "\n")
    wp, wd, wh, wv, wq = [], [], [], [], []
    for i, (a, b, c, d) in enumerate(qc):
        okp, pp = warp_feasible(a, b, c, d, 0)
        okd, pd = warp_feasible(a, b, c, d, 1)
        okv = wvrr_wanted(a, b, c, d) and pd["peak"] <= WARP_PEAK_MAX
        okq = okp and pvrr_wanted(a, b, c, d)
        wq.append(okq)
        okh = max(a, b, c, d) <= 1
        ph = warp_program(a, b, c, d, 2) if okh else None
        wp.append(okp)
        wd.append(okd)
        wh.append(okh)
        wv.append(okv)
        if (a, b, c, d) in COOP_CLASSES and not okp and not okd and not okv:
            continue
        with _Out(os.path.join(here, "gen", f"k_eri_{i:02d}.cu")) as f:
            f.write("// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.\n")
            f.write(f"// Kernels of class ({a}{b}|{c}{d}).\n")
            f.write('#include "../qx_warp.cuh"\n')
            f.write("using namespace qx;\n")
            if (a, b, c, d) not in COOP_CLASSES:
                f.write(f"QX_DEFINE_LAUNCH({i}, {a}, {b}, {c}, {d})\n")
            if okp:
                f.write(gen_warp_code(i, a, b, c, d, 0, pp, want_wvrr=okq) + "\n")
            if okd or okv:
                f.write(gen_warp_code(i, a, b, c, d, 1, pd, want_warp=okd, want_wvrr=okv) + "\n")
            if okh:
                f.write(gen_warp_code(i, a, b, c, d, 2, ph) + "\n")
    with _Out(os.path.join(here, "gen", "warp_index.cuh")) as f:
        f.write("// Generated by quax_b200/csrc/gen_eri.py -- do not edit by hand.\n#pragma once\n")
        f.write("#define QX_CLASS_WARP_PLAIN {" + ", ".join("1" if x else "0" for x in wp) + "}\n")
        f.write("#define QX_CLASS_WARP_DERIV {" + ", ".join("1" if x else "0" for x in wd) + "}\n")
        f.write("#define QX_FOR_EACH_WARP_PLAIN(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(wp) if x) + "\n")
        f.write("#define QX_FOR_EACH_WARP_DERIV(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(wd) if x) + "\n")
        f.write("#define QX_CLASS_WVRR {" + ", ".join("1" if x else "0" for x in wv) + "}\n")
        ds = [okd_ and okv_ for okd_, okv_ in zip(wd, wv)]
        f.write("#define QX_CLASS_DSPLIT {" + ", ".join("1" if x else "0" for x in ds) + "}\n")
        f.write("#define QX_FOR_EACH_DSPLIT(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(ds) if x) + "\n")
        f.write("#define QX_CLASS_PVRR {" + ", ".join("1" if x else "0" for x in wq) + "}\n")
        f.write("#define QX_FOR_EACH_PVRR(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(wq) if x) + "\n")
        f.write("#define QX_FOR_EACH_WVRR(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(wv) if x) + "\n")
        f.write("#define QX_CLASS_WARP_DERIV2 {" + ", ".join("1" if x else "0" for x in wh) + "}\n")
        f.write("#define QX_FOR_EACH_WARP_DERIV2(X) " + " ".join(f"X({i:02d})" for i, x in enumerate(wh) if x) + "\n")
    with _Out(os.path.join(here, "gen", "der_tables.cuh")) as f:
        f.write(gen_coop_deriv(list(enumerate(qc))))
    gen_rys(here, lmax)


if __name__ == "__main__":
    main()
