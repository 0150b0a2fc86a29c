"""Nuclear-derivative index bookkeeping, as the reference numbers it.

Mirrors quax/utils.py:39-70 (how_many_derivs, get_deriv_vec_idx) and the C++ helpers
quax/integrals/utils.h:100-172 (cartesian_product, process_deriv_vec,
how_many_derivs, generate_multi_index_lookup).  The numbering is the reference's:
unique derivatives of order k with respect to 3N coordinates are the
combinations with repetition of range(3N) taken k at a time, in lexicographic
order; a derivative vector (length 3N, entry i = how many times coordinate i is
differentiated) maps to the rank of its sorted multiset in that order.  The rank
is computed here in closed form instead of by enumeration.
"""
from __future__ import annotations

from itertools import product
from math import comb
from typing import List, Sequence, Tuple

import numpy as np


def how_many_derivs(k: int, n: int) -> int:
    """Unique Cartesian derivatives of order n for k atoms: C(3k + n - 1, n)."""
    return comb(3 * k + n - 1, n) if n > 0 else 1


def generate_multi_index_lookup(nparams: int, order: int) -> List[List[int]]:
    """Combinations with repetition of range(nparams), lexicographic."""
    out: List[List[int]] = []

    def rec(start: int, cur: List[int]):
        if len(cur) == order:
            out.append(list(cur))
            return
        for j in range(start, nparams):
            cur.append(j)
            rec(j, cur)
            cur.pop()

    rec(0, [])
    return out


def multiset_rank(sorted_idx: Sequence[int], nparams: int) -> int:
    """Rank of a non-decreasing index tuple among all such tuples of its length
    (lexicographic): for position i, count the tuples that agree before i and
    carry a smaller value at i -- with value v there, the remaining k-i-1
    positions draw from [v, nparams), C(nparams - v + k - i - 2, k - i - 1) ways."""
    k = len(sorted_idx)
    r = 0
    prev = 0
    for i, c in enumerate(sorted_idx):
        for v in range(prev, c):
            r += comb(nparams - v + k - i - 2, k - i - 1)
        prev = c
    return r


def get_deriv_vec_idx(deriv_vec) -> int:
    """Flattened upper-triangle index of a derivative vector (quax/utils.py:49-70)."""
    dv = np.asarray(deriv_vec, dtype=int).reshape(-1)
    idx = [i for i, m in enumerate(dv) for _ in range(int(m))]
    return multiset_rank(idx, dv.shape[0])


def process_deriv_vec(deriv_vec) -> Tuple[List[int], List[int]]:
    """deriv_vec -> (atoms, coordinates) with multiplicity (utils.h:116-128)."""
    atoms, coords = [], []
    for i, m in enumerate(deriv_vec):
        for _ in range(int(m)):
            atoms.append(i // 3)
            coords.append(i % 3)
    return atoms, coords


def cartesian_product(sets: Sequence[Sequence[int]]) -> List[List[int]]:
    """All picks of one element per set, first set varying slowest (utils.h:100-114)."""
    return [list(t) for t in product(*sets)]
