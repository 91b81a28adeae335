"""CPU restatement of libcudf's distinct rows and distinct-key hash join --
TEST INFRASTRUCTURE ONLY (the parity checker of tests/test_*distinct*.py);
the product never imports it.

Restates:
  * row equality of stream compaction: columns compared element-wise, NaNs
    equal under nan_equality::ALL_EQUAL and unequal under UNEQUAL, -0.0 ==
    +0.0, nulls equal under null_equality::EQUAL and a row holding a null
    distinct under UNEQUAL (src/stream_compaction/distinct_helpers.hpp:52,
    table/experimental/row_operators.cuh:1285-1312);
  * distinct_count(table, nulls_equal) (stream_compaction.hpp:422-424,
    src/stream_compaction/distinct_count.cu): the number of classes, NaNs equal;
  * distinct_indices(keep) (stream_compaction.hpp:311-317,
    src/stream_compaction/distinct.cu): per class its first (KEEP_FIRST,
    KEEP_ANY here), last (KEEP_LAST) row, or for KEEP_NONE the rows of
    single-row classes;
  * distinct_hash_join inner / left join (join.hpp:475-533,
    src/join/distinct_hash_join.cu): probe rows paired with the build row of
    an equal key (nulls match only under EQUAL; NaN matches NaN).
Rows are given as lists of (values ndarray, valid ndarray or None) columns.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def _canon(v, is_float: bool):
    if is_float:
        f = float(v)
        if math.isnan(f):
            return ("nan",)
        return 0.0 if f == 0.0 else f
    return v.item() if hasattr(v, "item") else v


def row_keys(cols: Sequence[Tuple[np.ndarray, Optional[np.ndarray]]], nulls_equal: bool = True,
             nans_equal: bool = True) -> List[object]:
    """One hashable key per row; a row distinct on its own gets a unique key."""
    n = len(cols[0][0]) if cols else 0
    out = []
    for r in range(n):
        parts = []
        alone = False
        for vals, valid in cols:
            ok = valid is None or bool(valid[r])
            if not ok:
                if not nulls_equal:
                    alone = True
                parts.append(("null",))
                continue
            is_f = vals.dtype.kind == "f"
            c = _canon(vals[r], is_f)
            if is_f and c == ("nan",) and not nans_equal:
                alone = True
            parts.append(c)
        out.append(("alone", r) if alone else tuple(parts))
    return out


def distinct_count(cols, nulls_equal: bool = True) -> int:
    return len(set(row_keys(cols, nulls_equal, True)))


def distinct_indices(cols, keep: int = 0, nulls_equal: bool = True, nans_equal: bool = True) -> np.ndarray:
    """keep: 0 ANY (first row here), 1 FIRST, 2 LAST, 3 NONE; sorted indices."""
    first: Dict[object, int] = {}
    last: Dict[object, int] = {}
    count: Dict[object, int] = {}
    for r, k in enumerate(row_keys(cols, nulls_equal, nans_equal)):
        first.setdefault(k, r)
        last[k] = r
        count[k] = count.get(k, 0) + 1
    if keep == 2:
        rows = last.values()
    elif keep == 3:
        rows = [first[k] for k, c in count.items() if c == 1]
    else:
        rows = first.values()
    return np.sort(np.fromiter(rows, dtype=np.int64, count=len(rows)))


def distinct_join(build, probe, nulls_equal: bool = True, left: bool = False):
    """inner: sorted (build, probe) pairs; left: build row (or INT32_MIN) per probe row."""
    bk = row_keys(build, nulls_equal, True)
    table: Dict[object, int] = {}
    for r, k in enumerate(bk):
        if isinstance(k, tuple) and len(k) == 2 and k[0] == "alone":
            continue
        table.setdefault(k, r)
    pk = row_keys(probe, nulls_equal, True)
    if left:
        return np.array([table.get(k, -(2 ** 31)) for k in pk], dtype=np.int64)
    pairs = sorted((table[k], r) for r, k in enumerate(pk) if k in table)
    return np.array(pairs, dtype=np.int64).reshape(-1, 2)
