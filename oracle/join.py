"""Hash joins restated on the CPU (dictionaries of row keys).

TEST INFRASTRUCTURE ONLY: the parity checker for libgbx's gbx_hash_join
(tests/).  Nothing in the product imports it.

Semantics (cudf::inner_join / left_join / full_join, join.hpp:107-190,
join/join.cu:33-118; left_semi_join / left_anti_join, join/semi_join.cu):
rows match when their keys are equal -- column by column, a STRUCT by its
validity and then its members (row_operators.cuh:1456-1500), NaN equal to
NaN and -0.0 to +0.0 (the nan-equal physical comparator, :1285-1312).  Under
null_equality::EQUAL nulls are equal at every level; under UNEQUAL a null
compares unequal to everything, so a row holding a null anywhere in its key
matches no row.  Results are sets of (left row, right row) pairs, None
standing for cudf::JoinNoneValue.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from cudf_b200._abi import JoinKind, NullEquality, TypeId
from oracle.oracle import HostCol
from oracle.structs import leaves


def _cell(v, tid):
    if tid == TypeId.STRING:
        return v
    if isinstance(v, (float, np.floating)):
        f = float(v)
        if math.isnan(f):
            return ("nan",)
        return 0.0 if f == 0.0 else f
    if isinstance(v, (bool, np.bool_)):
        return bool(v)
    return int(v)


def row_keys(keys: Sequence[HostCol]) -> Tuple[List[tuple], np.ndarray]:
    """Each row's key as a tuple of (valid, value) per leaf, and whether the
    row holds a null anywhere in its key."""
    n = keys[0].size if keys else 0
    lv = []
    for k in keys:
        lv += leaves(k, n)
    any_null = np.zeros(n, dtype=bool)
    cols = []
    for leaf in lv:
        any_null |= ~leaf.valid
        if leaf.values is None:
            cols.append([(bool(ok), None) for ok in leaf.valid])
        else:
            cols.append([(True, _cell(v, leaf.type_id)) if ok else (False, None)
                         for v, ok in zip(leaf.values, leaf.valid)])
    rows = [tuple(c[r] for c in cols) for r in range(n)]
    return rows, any_null


def hash_join(left: Sequence[HostCol], right: Sequence[HostCol], nulls_equal=NullEquality.EQUAL,
              kind=JoinKind.INNER) -> List[Tuple[Optional[int], Optional[int]]]:
    """The join's (left row, right row) pairs, sorted (semi / anti: (left
    row, None))."""
    lk, lnull = row_keys(left)
    rk, rnull = row_keys(right)
    unequal = nulls_equal == NullEquality.UNEQUAL
    table: Dict[tuple, List[int]] = {}
    for r, key in enumerate(rk):
        if unequal and rnull[r]:
            continue
        table.setdefault(key, []).append(r)
    out: List[Tuple[Optional[int], Optional[int]]] = []
    matched = set()
    for l, key in enumerate(lk):
        hits = [] if (unequal and lnull[l]) else table.get(key, [])
        if kind == JoinKind.LEFT_SEMI:
            if hits:
                out.append((l, None))
            continue
        if kind == JoinKind.LEFT_ANTI:
            if not hits:
                out.append((l, None))
            continue
        for r in hits:
            out.append((l, r))
            matched.add(r)
        if not hits and kind in (JoinKind.LEFT, JoinKind.FULL):
            out.append((l, None))
    if kind == JoinKind.FULL:
        out += [(None, r) for r in range(len(rk)) if r not in matched]
    return sorted(out, key=lambda p: (-1 if p[0] is None else p[0], -1 if p[1] is None else p[1]))
