"""Invariants of the kernel generator (host only): the chunked derivative programs
cover every accumulator target exactly once, each chunk's estimated live set fits
the budget, the item -> accumulator map of the split-mode kernels is a bijection
onto the cooperative layout, and the type-generic recurrences emit no FP64-only
literals (so the FP32 instantiation stays FP32)."""
import os
import re
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "quax_b200", "csrc"))
import gen_eri as G  # noqa: E402


@pytest.mark.parametrize("cls", [(1, 1, 1, 1), (2, 1, 1, 1), (2, 0, 2, 0)])
def test_chunked_derivative_program(cls):
    tl, spaces = G._warp_targets(*cls, 1)
    budget = G.WARP_LIVE_BUDGET[1]
    order, chunks = G._plan_targets(tl, budget)
    assert sorted(map(str, order)) == sorted(map(str, tl))
    assert chunks[0][0] == 0 and chunks[-1][1] == len(order)
    assert all(a < b for a, b in chunks) and all(chunks[k][1] == chunks[k + 1][0] for k in range(len(chunks) - 1))
    if len(chunks) > 1:
        assert all(G._chunk_cost(order[a:b])[1] <= budget for a, b in chunks)
    p = G.warp_program(*cls, 1)
    nacc = sum(sp.size for sp in spaces.values())
    assert p["nitem"] == nacc
    vm = [v for v in p["vmap"] if v != 0xFFFF]
    assert sorted(vm) == list(range(nacc))
    assert len(p["vmap"]) == p["nitem_pad"] and p["nitem_pad"] % 16 == 0


def test_type_generic_literals():
    p = G.warp_program(2, 1, 1, 0, 1)
    body = "\n".join(ln for ln in p["lines"] if not ln.lstrip().startswith("stg["))  # staging is FP64
    assert "const double v" not in body  # values are declared with the template type T
    # numeric literals in the recurrences are wrapped as T(...)
    bare = re.findall(r"(?<![\w(])\d+\.\d+(?!\))", body)
    assert not bare, bare[:5]
