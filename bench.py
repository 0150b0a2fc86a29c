#!/usr/bin/env python3
"""Headline benchmark: FP64 electron-repulsion integrals on B200.

Workload (one "step"): every Schwarz-screened 8-fold-unique contracted shell
quartet of a seeded synthetic molecule -- 10 atoms uniform in a 12-bohr cube
(minimum separation 1.8 bohr), Z in {1,6,8}, heavy atoms s,s,s,p,p,d and H s,s,p,
K ~ U{1..8} primitives per shell, exponents log-uniform in [0.08, 5e3], Schwarz
threshold 1e-12, Cartesian shells (the reference's convention) -- evaluated in
FP64 through the library's device path, with inputs resident in HBM.

  value   unique quartets / s over all ranks (replicas: one molecule per GPU)
  e2e     the same through the reference-facing C ABI with host buffers:
          qx_initialize (shells H2D) -> qx_compute_2e_int into pinned host memory
          (dense n^4 D2H, the reference's return convention) -> qx_finalize
  parity  the timed output against the CPU oracle, every quartet
  gradient_headline
          seconds per evaluation of sum Gamma dG/dR by the adjoint kernel and by
          the plain derivative-tensor path (derivative integrals materialised tile
          by tile as (3N, tile) tensors, then contracted): 10 and 30 atoms in full,
          the 60-atom workload with f shells through a cost-balanced 1/64 shard

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun (N>1) each rank runs its own replica; the max over ranks is used.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "HF geom-gradient s/eval (adjoint vs plain ERI-deriv) at 1e-8 Eh/bohr; quartets/s"
WORKLOAD = "eri10"
THR = 1e-12
# DRAM traffic of a class's dominant kernel from an ncu capture of this workload
# (dram__bytes_read.sum + dram__bytes_write.sum), with the capture it comes from
TRAFFIC_FROM_PROFILE = {
    (2, 2, 2, 1): {"bytes": 29.21e6, "source": "ncu capture in profiles/k_gvrr_p19_eri10.md (split VRR kernel "
                                               "of the class, one launch)"},
}


def workload_desc(b, extra=None):
    d = {
        "workload": "10-atom synthetic molecule, l<=2, K 1-8, Schwarz 1e-12, full unique FP64 ERI (seed 0)",
        "natom": b.natom,
        "nshell": b.nshell,
        "nbf": b.nbf(),
        "shells": "cartesian",
        "schwarz_tol": THR,
        "l2": "flushed between steps (256 MiB write); inputs are L2-resident pair data",
        "parallelism": "replicas (one molecule per GPU, no exchange)",
    }
    if extra:
        d.update(extra)
    return d


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ------------------------------------------------------------------ clocks ----
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms",
                 "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for ln in fh:
                p = [x.strip() for x in ln.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ our arm ---
def fp64_peak_tflops():
    lib = ctypes.CDLL(os.path.join(ROOT, "quax_b200", "libqx_peaks.so"))
    lib.qx_fma_peak_tflops.restype = ctypes.c_double
    lib.qx_fma_peak_tflops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qx_fma_peak_tflops(1, 2000, 1)
    return max(lib.qx_fma_peak_tflops(1, 20000, 3) for _ in range(3))


def cpu_baseline_eri(basis, target_s=12.0):
    """Oracle (CPU port, all host threads) on a bounded sample of the same quartets."""
    from oracle import api

    ob = api.OracleBasis(basis)
    K, kmax = api.schwarz(ob)
    # calibrate: a small sample, then a sample sized for ~target_s seconds
    t = time.perf_counter()
    n0, _ = api.unique_sample(ob, THR, 400, 0, K=K, kmax=kmax)
    dt0 = max(time.perf_counter() - t, 1e-3)
    rate0 = n0 / dt0
    total = api.count_unique(ob, THR)
    stride = max(1, int(total / max(rate0 * target_s, 1.0)))
    t = time.perf_counter()
    n, _ = api.unique_sample(ob, THR, stride, 1 % stride, K=K, kmax=kmax)
    dt = time.perf_counter() - t
    return {"value": n / dt, "unit": "quartets/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"every {stride}-th of {total} screened unique quartets ({n} quartets, {dt:.1f} s; "
                      f"Schwarz pass excluded); C/OpenMP oracle, FP64"}


def parity_vs_oracle(eng, b, out):
    """The timed output against the oracle: every screened unique quartet's block
    (class by class, list order) compared with the oracle's block of the same
    canonical shell quartet (oracle on all host threads)."""
    import numpy as np
    import torch

    from oracle import api

    ob = api.OracleBasis(b)
    base, err, err_scaled, nq_tot = 0, 0.0, 0.0, 0
    t0 = time.perf_counter()
    for c in eng.class_info():
        nq = c["nq"]
        ncomp = int(np.prod([(l + 1) * (l + 2) // 2 for l in c["l"]]))
        if nq:
            ref = torch.from_numpy(api.quartet_blocks(ob, eng.class_quartets(c["cls"]))).cuda()
            d = (out[base:base + nq * ncomp].view(ncomp, nq).T - ref).abs()
            err = max(err, float(d.max()))
            err_scaled = max(err_scaled, float((d.amax(dim=1) / ref.abs().amax(dim=1).clamp(min=1.0)).max()))
            nq_tot += nq
        base += nq * ncomp
    return {"max_abs_err": err, "max_err_over_block_scale": err_scaled, "quartets_checked": nq_tot,
            "oracle": "C/OpenMP Obara-Saika/Head-Gordon-Pople restatement (oracle/eri_oracle.c), FP64",
            "block_scale": "max(1, largest |integral| of the quartet's block)",
            "oracle_s": time.perf_counter() - t0}


def run_ours(args):
    import numpy as np
    import torch

    from quax_b200.basis import config_spec, synthetic_molecule
    from quax_b200.integrals import _lib
    from quax_b200.integrals.engine import EriEngine

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    mol, b = synthetic_molecule(config_spec(WORKLOAD), 0)
    eng = EriEngine(b, THR)
    # engine per class chosen by the library's autotuner (outside the timed region)
    t_tune = time.perf_counter()
    eng.autotune(plain=True, deriv=not args.no_grad and not args.no_extras)
    t_tune = time.perf_counter() - t_tune
    nq = eng.unique_quartets()
    out = torch.empty(eng.unique_size(), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    info = eng.class_info()
    total_flops = sum(c["flops"] for c in info)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if args.no_extras:
        torch.cuda.profiler.start()  # profiling runs: the steps only (ncu --profile-from-start off)
    for _ in range(args.warmup):
        eng.eri_unique(out)
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier()
        for s in range(args.steps):
            flush.zero_()
            ev[s][0].record()
            eng.eri_unique(out)
            ev[s][1].record()
        barrier()
    clocks = clk.summary()
    ms = sum(a.elapsed_time(b_) for a, b_ in ev)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * nq / (ms_per_step * 1e-3)
    # our kernels per step: one per class with quartets, two for split-mode classes
    # (primitive-chunk VRR + HRR)
    cfg = eng.engine_config()
    launches = sum(2 if cfg["%d%d%d%d" % c["l"]][0] == "wsplit" else 1 for c in info if c["nq"] > 0) * args.steps

    if args.no_extras:
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "quartets/s", "ms_per_step": ms_per_step,
                              "note": "--no-extras (profiling run)"}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    # roofline of the dominant kernel: time every class launch alone (events on the
    # launching stream), pick the longest, FLOPs from the op-count table
    s = torch.cuda.current_stream()
    per = []
    for c in info:
        if c["nq"] == 0:
            continue
        eng.eri_unique_class(c["cls"], out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        reps = 3
        e0.record(s)
        for _ in range(reps):
            eng.eri_unique_class(c["cls"], out)
        e1.record(s)
        torch.cuda.synchronize()
        per.append((e0.elapsed_time(e1) / reps, c))
    per.sort(key=lambda x: -x[0])
    dom_ms, dom = per[0]
    peak = fp64_peak_tflops()
    achieved = dom["flops"] / (dom_ms * 1e-3) / 1e12
    roofline = {
        "bound": "fp64",
        "kernel": f"class ({dom['l'][0]}{dom['l'][1]}|{dom['l'][2]}{dom['l'][3]}) ERI kernel",
        "achieved": achieved,
        "peak": peak,
        "unit": "TFLOP/s",
        "frac": achieved / peak if peak > 0 else None,
        "peak_source": "measured FP64 FMA probe (libqx_peaks.so), not in MEASURED_PEAKS.json",
        # DRAM bytes per launch of the dominant kernel: copied from one ncu capture
        # of the same workload (not measured by this run), null for other classes
        "traffic": TRAFFIC_FROM_PROFILE.get(tuple(dom["l"]), {}).get("bytes"),
        "traffic_unit": "bytes per launch",
        "traffic_source": TRAFFIC_FROM_PROFILE.get(tuple(dom["l"]), {}).get("source",
                                                                           "no ncu capture of this class's kernel"),
        "step_achieved_tflops": total_flops / (ms_per_step * 1e-3) / 1e12,
        "dominant_share_of_serial_sum": dom_ms / sum(p[0] for p in per),
    }

    # end to end through the reference-facing C ABI with host buffers
    lib = _lib.load()
    fl = b.flat()
    coords = np.ascontiguousarray(b.atom_coords().reshape(-1))
    n = eng.nbf
    host = torch.empty(n**4, dtype=torch.float64, pin_memory=True)
    h2d = coords.nbytes + sum(fl[k].nbytes for k in ("l", "nprim", "atom", "exps", "coefs"))

    def e2e_step():
        h = ctypes.c_void_p()
        _lib.check(lib.qx_initialize(b.natom, _lib.dptr(coords), b.nshell, _lib.iptr(fl["l"]), _lib.iptr(fl["nprim"]),
                                     _lib.iptr(fl["atom"]), _lib.dptr(fl["exps"]), _lib.dptr(fl["coefs"]), 0, THR,
                                     ctypes.byref(h)), "qx_initialize")
        _lib.check(lib.qx_compute_2e_int(h, ctypes.c_void_p(host.data_ptr()), 0, ctypes.c_void_p(0)),
                   "qx_compute_2e_int")
        lib.qx_finalize(h)

    e2e_step()
    barrier()
    e2e_steps = max(3, min(args.steps, 5))
    ts = []
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        e2e_step()
        barrier()
        ts.append(time.perf_counter() - t0)
    e2e_s = statistics.median(ts)
    e2e = {"value": world * nq / e2e_s, "unit": "quartets/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(8 * n**4), "ms_per_step": e2e_s * 1e3,
           "ms_per_step_all": [round(t * 1e3, 2) for t in ts], "statistic": "median over steps (host wall clock)",
           "path": "qx_initialize + qx_compute_2e_int(host pinned n^4) + qx_finalize"}
    del host

    # the same molecule with spherical d shells (the synthetic workload's basis):
    # Cartesian kernels + the device solid-harmonic transform of every class
    from quax_b200.basis import Basis
    from quax_b200.integrals.spherical import SphericalEngine

    sph = SphericalEngine(Basis(b.shells, b.natom, True, b.name), THR)
    sph.cart.autotune(plain=True, deriv=False)
    sph.eri_unique()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        sph.eri_unique()
    e1.record()
    torch.cuda.synchronize()
    sph_ms = e0.elapsed_time(e1) / 3
    spherical = {"nbf": sph.nbf, "ms_per_step": sph_ms, "value": nq / (sph_ms * 1e-3), "unit": "quartets/s",
                 "path": "Cartesian unique kernels + per-class solid-harmonic transform kernel (qx_cart2sph_block)"}
    sph.close()

    grad = batched = None
    if not args.no_grad:
        grad = gradient_headline(eng, b, oracle_check=rank == 0)
        batched = batched_extras(args.batch)

    parity = parity_vs_oracle(eng, b, out) if rank == 0 else None
    cpu = cpu_baseline_eri(b) if rank == 0 else None
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "quartets/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded generator; no dataset)",
            "config": workload_desc(b, {"unique_quartets": nq, "primitive_quartets": sum(c["prims"] for c in info),
                                        "engines": "per class by qx_autotune (%.1f s, untimed)" % t_tune,
                                        "engine_config": eng.engine_config()}),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
            "parity": parity,
            "gradient_headline": grad,
            "batched_rhf": batched,
            "spherical": spherical,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _density(n, seed=0):
    """D = C C^T, C an n x n/4 matrix of iid N(0, 1/n) entries (the 30-atom
    workload's definition of Gamma's density)."""
    import numpy as np
    import torch

    rng = np.random.default_rng(seed)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, max(1, n // 4)))
    return torch.from_numpy(C @ C.T).cuda()


def _time_ms(fn, reps=1, warm=True):
    """Device time of fn() (CUDA events on the current stream; one warm-up call
    unless warm is False, for long calls whose kernels already ran)."""
    import torch

    if warm:
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _tile_engines(eng, D, shard=8, view=(0, 1)):
    """Per class, the fastest derivative engine among those the plain path can also
    use (warp kernels with 1 or 4 warps per quartet, Rys), timed in adjoint mode on
    a 1/shard cost-balanced shard of the lists, so the adjoint and the plain path
    below run the same derivative arithmetic."""
    import torch

    g = torch.zeros(3 * eng.natom, dtype=torch.float64, device="cuda")
    cfg = eng.engine_config()
    if view == (0, 1):
        eng.set_shard(0, shard)  # an unsharded handle is timed on a shard
    for c in eng.class_info():
        if not c["nq"] or cfg["%d%d%d%d" % c["l"]][2] in ("warp", "rys"):
            continue  # the autotuned engine has the tile epilogue already
        best = None
        for name, p in (("warp", 1), ("warp", 4), ("rys", 0)):
            try:
                eng.set_engine(c["cls"], deriv=name, deriv_param=p)
            except NotImplementedError:
                continue
            ms = _time_ms(lambda: eng.grad_adjoint_class(c["cls"], D, g))
            if best is None or ms < best[0]:
                best = (ms, name, p)
        eng.set_engine(c["cls"], deriv=best[1], deriv_param=best[2])
    if view == (0, 1):
        eng.set_shard(0, 1)


def _autotune_on_shard(eng, shard, plain=False):
    """Engines per class chosen by the autotuner on a 1/shard cost-balanced shard
    of the lists (the choices persist when the full lists are restored)."""
    eng.set_shard(0, shard)
    eng.autotune(plain=plain, deriv=True)
    eng.set_shard(0, 1)


def _adjoint_vs_plain(eng, D, reps=1, warm=True, unique=True, view=(0, 1)):
    """Adjoint gradient vs the plain derivative-tensor path on one handle: the
    adjoint with the autotuned engines, then both paths with the same per-class
    engines (the plain path materialises every derivative integral -- each image
    of the reference's (3N, n^4) tensor, tile by tile -- and contracts the tiles
    with Gamma; each derivative quartet is evaluated once)."""
    r = {"adjoint_autotuned_s": _time_ms(lambda: eng.grad_adjoint(D), reps, warm) * 1e-3}
    _tile_engines(eng, D, view=view)
    ga = eng.grad_adjoint(D)  # also warms the chosen engines
    r["adjoint_s"] = _time_ms(lambda: eng.grad_adjoint(D), reps, False) * 1e-3
    gp = eng.grad_plain(D, images=True)
    r["plain_s"] = _time_ms(lambda: eng.grad_plain(D, images=True), reps, False) * 1e-3
    if unique:
        r["plain_unique_elements_s"] = _time_ms(lambda: eng.grad_plain(D, images=False), reps, False) * 1e-3
    r["max_abs_diff_adjoint_vs_plain_Eh_per_bohr"] = float((ga - gp).abs().max())
    r["adjoint_speedup_vs_plain"] = r["plain_s"] / r["adjoint_s"]
    r["tile_engines"] = {k: v[2] for k, v in eng.engine_config().items()}
    return r, ga


def _hessian_column(eng, D, warm=True):
    import torch

    e0 = torch.zeros(3 * eng.natom, dtype=torch.float64)
    e0[0] = 1.0
    return _time_ms(lambda: eng.grad_adjoint_jvp(D, e0), 1, warm) * 1e-3


def gradient_headline(eng10, b10, oracle_check=True):
    """The headline quantity: s per evaluation of the HF-type gradient
    sum Gamma_ijkl d(ij|kl)/dR (Gamma = D_ij D_kl - 1/2 D_ik D_jl), adjoint kernel
    vs the plain FP64 derivative-tensor path, on the 10- and 30-atom workloads in
    full and on the 60-atom workload with f shells through a cost-balanced shard."""
    import numpy as np
    import torch

    from quax_b200.basis import config_spec, synthetic_molecule
    from quax_b200.integrals.engine import EriEngine

    out = {"gamma": "D_ij D_kl - 1/2 D_ik D_jl, D = C C^T, C n x n/4 iid N(0,1/n), seed 0",
           "plain_path": "first-derivative integrals of tiles of unique quartets materialised as (3N, tile) "
                         "tensors holding every image of each integral (the reference tensor's elements), "
                         "then one GEMV per tile with Gamma; each derivative quartet evaluated once"}
    # 10 atoms: error against the oracle over a contiguous eighth of every class
    D10 = _density(eng10.nbf)
    w10, _ = _adjoint_vs_plain(eng10, D10, reps=3)
    w10["hessian_column_jvp_s"] = _hessian_column(eng10, D10)
    if oracle_check:
        from oracle import api

        ob = api.OracleBasis(b10)
        eng10.set_shard(0, 8)
        err, gmax = 0.0, 0.0
        g = torch.zeros(3 * b10.natom, dtype=torch.float64, device="cuda")
        for c in eng10.class_info():
            if not c["nq"]:
                continue
            g.zero_()
            eng10.grad_adjoint_class(c["cls"], D10, g)
            ref = api.grad_quartets(ob, eng10.class_quartets(c["cls"]), D10.cpu().numpy(), 1.0, -0.5)
            err = max(err, float(np.abs(g.cpu().numpy() - ref).max()))
            gmax = max(gmax, float(np.abs(ref).max()))
        eng10.set_shard(0, 1)
        w10["max_abs_err_vs_oracle_Eh_per_bohr"] = err
        w10["oracle_sample"] = "per class, the contiguous eighth of its quartet list with the most primitives"
    out["workload_10_atoms"] = w10
    # 30 atoms (l <= 2), in full
    _, b30 = synthetic_molecule(config_spec("grad30"), 0)
    t0 = time.perf_counter()
    e30 = EriEngine(b30, THR)
    init30 = time.perf_counter() - t0
    D30 = _density(e30.nbf)
    _autotune_on_shard(e30, 8)
    w30, g64 = _adjoint_vs_plain(e30, D30, warm=True)
    w30.update({"natom": b30.natom, "nbf": e30.nbf, "unique_quartets": e30.unique_quartets(), "init_s": init30,
                "engines": "derivative engines autotuned on a 1/8 cost-balanced shard of the lists"})
    # mixed precision over the whole molecule: FP32 recurrences below a Schwarz
    # bound of 1e-6 (reorders the lists, so measured unsharded), error vs FP64
    e30.set_precision(1e-6)
    g32 = e30.grad_adjoint(D30)
    w30["mixed_precision"] = {"bound": 1e-6, "adjoint_s": _time_ms(lambda: e30.grad_adjoint(D30), 1, False) * 1e-3,
                              "max_abs_dgrad_vs_fp64_Eh_per_bohr": float((g32 - g64).abs().max())}
    e30.close()
    out["workload_30_atoms"] = w30
    out["workload_60_atoms_f"] = gradient_60_atoms()
    return out


def gradient_60_atoms(S=128):
    """The 60-atom workload with f shells (K 1-3, exponents 0.2-5 on the heavy
    atoms): every timing on rank S/2 of an S-way cost-balanced shard (each class
    keeps a contiguous range of its quartets of about 1/S of its primitive work),
    scaled by S to an s/eval estimate -- the full evaluation runs minutes."""
    import torch

    from quax_b200.basis import config_spec, synthetic_molecule
    from quax_b200.integrals.engine import EriEngine

    _, b = synthetic_molecule(config_spec("mixed60"), 0)
    t0 = time.perf_counter()
    eng = EriEngine(b, THR)
    init = time.perf_counter() - t0
    info = eng.class_info()
    r = {"natom": b.natom, "nbf_cartesian": eng.nbf, "unique_quartets": eng.unique_quartets(),
         "f_quartets": sum(c["nq"] for c in info if max(c["l"]) == 3),
         "primitive_quartets": sum(c["prims"] for c in info), "init_s": init,
         "sample": f"rank {S // 2} of {S} cost-balanced shards; times x {S}"}
    eng.set_shard(S // 2, S)
    eng.autotune(plain=True, deriv=True)
    D = _density(eng.nbf)
    r["jk_s_estimate"] = _time_ms(lambda: eng.jk(D)) * 1e-3 * S
    a, _ = _adjoint_vs_plain(eng, D, warm=False, unique=False, view=(S // 2, S))
    for k in ("adjoint_autotuned_s", "adjoint_s", "plain_s"):
        r[k.replace("_s", "_s_estimate")] = a[k] * S
    r["adjoint_speedup_vs_plain"] = a["adjoint_speedup_vs_plain"]
    r["max_abs_diff_adjoint_vs_plain_Eh_per_bohr (shard)"] = a["max_abs_diff_adjoint_vs_plain_Eh_per_bohr"]
    # one Hessian column (the JVP of the adjoint gradient along atom 0's x): only
    # the quartets with a centre on atom 0 contribute, a few per cent of each
    # list, so it is timed on a larger sample (1/16) than the gradient
    S2 = 16
    eng.set_shard(S2 // 2, S2)
    v = torch.zeros(3 * eng.natom, dtype=torch.float64, device="cuda")
    v[0] = 1.0
    r["hessian_column_jvp_s_estimate"] = _time_ms(lambda: eng.grad_adjoint_jvp(D, v), 1, False) * 1e-3 * S2
    r["hessian_column_sample"] = f"rank {S2 // 2} of {S2} cost-balanced shards; time x {S2}"
    eng.close()
    return r


def batched_extras(count: int, iterations: int = 20):
    """Batched RHF: `count` Gaussian-displaced geometries (sigma 0.05 bohr) of one
    12-atom synthetic molecule, J/K of the whole batch replayed from one CUDA graph
    per SCF iteration (incremental builds from the density change with density
    screening at 1e-12, full rebuild every 8 iterations), then the analytic
    gradients."""
    import torch

    from quax_b200.basis import SyntheticSpec, synthetic_molecule
    from quax_b200.methods.batch import BatchedRHF, displaced_geometries

    spec = SyntheticSpec(natom=12)
    mol0, b0 = synthetic_molecule(spec, 0)
    mols = displaced_geometries(mol0, count, 0.05, seed=1)
    bases = [b0.with_coords(m.coords) for m in mols]
    t0 = time.perf_counter()
    br = BatchedRHF(mols, bases, ints_tol=THR, incremental=1e-12, rebuild_every=8)
    nq = sum(m.eng.unique_quartets() for m in br.mols)
    # eager J/K of the batch, for comparison with the graph replay
    br._jk_all()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    br._jk_all()
    e1.record()
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1)
    t1 = time.perf_counter()
    E, t_jk = br.scf(iterations=iterations, use_graph=True)
    t2 = time.perf_counter()
    G = br.gradients()
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    br.close()
    return {"molecules": count, "natom": mol0.natom, "nbf": b0.nbf(), "unique_quartets_per_jk": nq,
            "scf_iterations": iterations, "setup_s": t1 - t0, "scf_s": t2 - t1,
            "jk_graph_ms_per_iteration (incremental, density-screened builds)": t_jk / iterations * 1e3,
            "full_jk_eager_ms": eager_ms, "full_jk_quartets_per_s": nq / (eager_ms * 1e-3), "gradients_s": t3 - t2,
            "energy_spread_Eh": float(max(E) - min(E)),
            "max_abs_gradient": float(max(abs(g).max() for g in G))}


def config4_run(args):
    """The batched uneven workload: `--config4` molecules (64 by default) of 3-40
    atoms (sizes drawn from seed 0, molecule i generated with seed i), each with
    FP64 RHF for 20 iterations -- every iteration's J/K of the whole batch
    replayed from one CUDA graph, incremental density-screened builds with a full
    rebuild every 8 iterations -- then the adjoint gradients.  Prints one JSON line."""
    import numpy as np
    import torch

    from quax_b200.basis import SyntheticSpec, synthetic_molecule
    from quax_b200.methods.batch import BatchedRHF

    sizes = np.random.default_rng(0).integers(3, 41, size=args.config4)
    mols, bases = [], []
    for i, k in enumerate(sizes):
        m, b = synthetic_molecule(SyntheticSpec(natom=int(k)), i)
        mols.append(m)
        bases.append(b)
    t0 = time.perf_counter()
    br = BatchedRHF(mols, bases, ints_tol=THR, incremental=1e-12, rebuild_every=8)
    nq = sum(m.eng.unique_quartets() for m in br.mols)
    br._jk_all()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    br._jk_all()
    e1.record()
    torch.cuda.synchronize()
    jk_ms = e0.elapsed_time(e1)
    t1 = time.perf_counter()
    E, t_jk = br.scf(iterations=20, use_graph=True)
    t2 = time.perf_counter()
    G = br.gradients()
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    br.close()
    print(json.dumps({"workload": f"{len(sizes)} molecules of 3-40 atoms (l<=2, Cartesian), FP64 RHF 20 iterations "
                                  "+ adjoint gradients", "natoms": [int(k) for k in sizes],
                      "nbf_total": int(sum(b.nbf() for b in bases)), "unique_quartets_per_full_jk": nq,
                      "setup_s": t1 - t0, "full_jk_eager_ms": jk_ms, "full_jk_quartets_per_s": nq / (jk_ms * 1e-3),
                      "scf_s": t2 - t1, "jk_graph_ms_per_iteration (incremental, density-screened builds)":
                      t_jk / 20 * 1e3, "gradients_s": t3 - t2,
                      "max_abs_gradient": float(max(abs(g).max() for g in G))}), flush=True)


def run_grad_only(args):
    """Adjoint gradient of the workload only (profiling aid; prints its timing).
    With --profile-f: an 8-atom synthetic molecule with f shells on the heavy
    atoms (the 60-atom workload's shell mix at a size a profiler replays quickly),
    whose gradient is dominated by the Rys kernels of the f classes."""
    import numpy as np
    import torch

    from quax_b200.basis import SyntheticSpec, config_spec, synthetic_molecule
    from quax_b200.integrals.engine import EriEngine

    if args.profile_f:
        mol, b = synthetic_molecule(SyntheticSpec(natom=8, f_shell=True), 0)
    else:
        mol, b = synthetic_molecule(config_spec(WORKLOAD), 0)
    eng = EriEngine(b, THR)
    eng.autotune(plain=False, deriv=True)
    n = eng.nbf
    rng = np.random.default_rng(0)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, n // 4))
    D = torch.from_numpy(C @ C.T).cuda()
    torch.cuda.profiler.start()  # profiled region: the warm-up and timed gradients only
    for _ in range(args.warmup):
        eng.grad_adjoint(D)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        eng.grad_adjoint(D)
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    # per class (outside the profiled region): one event-timed evaluation and the
    # algorithmic first-derivative FLOPs qx_class_info reports
    g = torch.zeros(3 * eng.natom, dtype=torch.float64, device="cuda")
    classes = {}
    for c in eng.class_info():
        if not c["nq"]:
            continue
        e0.record()
        eng.grad_adjoint_class(c["cls"], D, g)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        classes["%d%d%d%d" % c["l"]] = {"ms": t, "gflop": c["flops_deriv"] * 1e-9,
                                        "tflops": c["flops_deriv"] / (t * 1e-3) * 1e-12}
    print(json.dumps({"adjoint_ms": ms, "note": "--profile-grad", "engine_config": eng.engine_config(),
                      "classes": classes}), flush=True)


# ------------------------------------------------------------- reference arm ---
def run_reference(args):
    """The reference's CPU path for this workload on the host cores.  Libint (the
    reference's engine) cannot be built or imported on this image, so the timed CPU
    implementation is the oracle port (C/OpenMP restatement of the same algorithm
    and screening), each step a bounded sample of the workload."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import api
    from quax_b200.basis import config_spec, synthetic_molecule

    mol, b = synthetic_molecule(config_spec(WORKLOAD), 0)
    ob = api.OracleBasis(b)
    K, kmax = api.schwarz(ob)
    total = api.count_unique(ob, THR)
    stride = 64
    for w in range(args.warmup):
        api.unique_sample(ob, THR, stride * 4, w % (stride * 4), K=K, kmax=kmax)
    t = time.perf_counter()
    done = 0
    for s in range(args.steps):
        n, _ = api.unique_sample(ob, THR, stride, s % stride, K=K, kmax=kmax)
        done += n
    dt = time.perf_counter() - t
    value = done / dt
    sample = (f"each step: every {stride}-th of {total} screened unique quartets (phase = step index); "
              f"{done} quartets in {dt:.1f} s; Schwarz pass excluded; oracle C/OpenMP port (Libint unavailable)")
    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator; no dataset)",
        "config": workload_desc(b, {"unique_quartets": total}),
        "cpu_baseline": {"value": value, "unit": "quartets/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-grad", action="store_true", help="skip the adjoint/plain gradient extras")
    ap.add_argument("--batch", type=int, default=32,
                    help="displaced geometries in the batched-RHF extra (the full workload is 256)")
    ap.add_argument("--profile-grad", action="store_true",
                    help="run only the adjoint gradient of the workload, warmup+steps times (for profiler runs)")
    ap.add_argument("--config4", type=int, default=0,
                    help="run only the batched uneven workload with this many molecules (64: the full one)")
    ap.add_argument("--profile-f", action="store_true",
                    help="with --profile-grad: an 8-atom molecule with f shells instead of the workload")
    ap.add_argument("--no-extras", action="store_true",
                    help="time the ERI steps only (for profiler runs): no roofline probe, e2e, gradient or CPU arm")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.profile_grad:
        run_grad_only(args)
    elif args.config4:
        config4_run(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
