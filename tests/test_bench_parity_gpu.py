"""The timed workload pinned to the oracle.

The benchmark's molecule exactly as bench.py builds it (10 synthetic atoms, seed 0,
l <= 2, K 1-8, exponents log-uniform in [0.08, 5e3], Schwarz 1e-12; 423,337 screened
unique quartets).  For every class, every engine and parameter the class can run
is forced through qx_set_engine (the autotuner's choices included), and:

  * qx_eri_unique_class is compared element by element with the oracle's block of
    the same canonical shell quartet, in the same list order (reference semantics
    libint_interface.cc:486-647), to 2e-12 x max(1, largest |integral| of the
    quartet's block).  The 1e-12 plain-path bar is doubled because the oracle
    itself carries ~1e-12 rounding on this workload: on quartet (38,5|38,5) its
    (xx,xx|xx,xx) element differs from a 40-digit evaluation by 1.03e-12 (the
    Rys engine's by 1.2e-15) -- Obara-Saika recurrences on (dd|dd) quartets with
    exponents spanning four decades cancel that much;
  * qx_grad_adjoint_class on a contiguous eighth of every class's list (the
    quartets with the most primitives: the lists are sorted by primitive count)
    is compared with the oracle's contribution of the same quartets (1e-9
    absolute scaled by max(1, |g|), the gradient bar).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

PLAIN = [("sl", lg) for lg in range(6)] + [("warp", 1), ("warp", 4), ("coop", 0), ("wsplit", 1), ("rys", 0)]
DERIV = [("warp", 1), ("warp", 4), ("wvrr", 0), ("dsplit", 0), ("coop", 0), ("rys", 0), ("rys", 1)]


@pytest.fixture(scope="module")
def bench_case(oracle_lib):
    from quax_b200.basis import config_spec, synthetic_molecule
    from quax_b200.integrals.engine import EriEngine

    _, b = synthetic_molecule(config_spec("eri10"), 0)
    eng = EriEngine(b, 1e-12)
    ob = oracle_lib.OracleBasis(b)
    yield eng, b, ob
    eng.close()


def _layout(eng):
    base, out = 0, {}
    for c in eng.class_info():
        ncomp = int(np.prod([(l + 1) * (l + 2) // 2 for l in c["l"]]))
        out[c["cls"]] = (base, c["nq"], ncomp, c["l"])
        base += c["nq"] * ncomp
    return out


def test_bench_unique_every_engine(bench_case, oracle_lib):
    eng, b, ob = bench_case
    assert eng.unique_quartets() == 423337
    lay = _layout(eng)
    out = torch.zeros(eng.unique_size(), dtype=torch.float64, device="cuda")
    ntried = 0
    for cls, (base, nq, ncomp, l) in lay.items():
        if not nq:
            continue
        ref = torch.from_numpy(oracle_lib.quartet_blocks(ob, eng.class_quartets(cls))).cuda()
        scale = ref.abs().amax(dim=1).clamp(min=1.0)  # per quartet
        view = out[base:base + nq * ncomp].view(ncomp, nq)
        for name, param in PLAIN:
            try:
                eng.set_engine(cls, plain=name, plain_param=param)
            except NotImplementedError:
                continue
            view.zero_()
            eng.eri_unique_class(cls, out)
            err = float(((view.T - ref).abs().amax(dim=1) / scale).max())
            assert err < 2e-12, (l, name, param, err)
            ntried += 1
    assert ntried >= 2 * len([1 for v in lay.values() if v[1]])


def test_bench_grad_every_engine(bench_case, oracle_lib):
    eng, b, ob = bench_case
    n = eng.nbf
    rng = np.random.default_rng(0)
    C = rng.normal(0.0, 1.0 / np.sqrt(n), size=(n, n // 4))
    D = C @ C.T
    Dt = torch.from_numpy(D).cuda()
    eng.set_shard(0, 8)
    try:
        g = torch.zeros(3 * b.natom, dtype=torch.float64, device="cuda")
        for c in eng.class_info():
            if not c["nq"]:
                continue
            ref = oracle_lib.grad_quartets(ob, eng.class_quartets(c["cls"]), D, 1.0, -0.5)
            tol = 1e-9 * max(1.0, np.abs(ref).max())
            for name, param in DERIV:
                try:
                    eng.set_engine(c["cls"], deriv=name, deriv_param=param)
                except NotImplementedError:
                    continue
                g.zero_()
                eng.grad_adjoint_class(c["cls"], Dt, g, 1.0, -0.5)
                err = float(np.abs(g.cpu().numpy() - ref).max())
                assert err < tol, (c["l"], name, param, err)
    finally:
        eng.set_shard(0, 1)
