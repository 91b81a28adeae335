"""Groups of keys the caller declares sorted, formed as the reference's sort
path forms them.

TEST INFRASTRUCTURE ONLY: the parity checker for libgbx's keys_are_sorted
path (tests/).  Nothing in the product imports it.

cudf::groupby::groupby(keys, null_policy, sorted::YES) aggregates on the sort
path (groupby/groupby.cu:197-221).  Its helper keeps the rows in their given
order (groupby/sort/sort_helper.cu:96-104) and starts a group wherever a row's
key differs from the row before it, nulls equal and NaNs equal
(sort_helper.cu:141-179, row_operators.cuh:1338).  Under null_policy EXCLUDE
with null keys the helper does not trust the order: it sorts the rows again,
stably, the rows holding a null key last, and cuts those off
(sort_helper.cu:64-71, 74-88, 106-133).  Each group's key is read at its first
row in that order (sort/groupby.cu: the keys gathered at the group offsets).

Here each row is labelled with its group's index in that order, the plain
oracle (oracle.groupby) aggregates by the label, and the result is put in
label order with the key columns read at each group's first row.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from cudf_b200._abi import NullPolicy, TypeId
from oracle import oracle as orc
from oracle.oracle import HostCol


def _key_rows(k: HostCol):
    """(valid, comparable values, NaN flags) of a key column's rows: floats
    with -0.0 as 0.0 and NaNs flagged, strings as str (null: ""),
    dictionaries as their indices."""
    s = slice(k.offset, k.offset + k.size)
    valid = np.ones(k.size, dtype=bool) if k.valid is None else np.asarray(k.valid, dtype=bool)[s]
    vals = k.values[s]
    nan = np.zeros(k.size, dtype=bool)
    if k.type_id == TypeId.STRING:
        vals = np.array(["" if v is None else v for v in vals], dtype=object)
    elif vals.dtype.kind == "f":
        nan = np.isnan(vals)
        vals = np.where(nan | (vals == 0), 0.0, vals).astype(vals.dtype)
    return valid, vals, nan


def _rows_differ(cols, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Row a[i]'s key differs from row b[i]'s (nulls equal, NaNs equal)."""
    diff = np.zeros(len(a), dtype=bool)
    for valid, vals, nan in cols:
        va, vb = valid[a], valid[b]
        both = va & vb
        same = (nan[a] == nan[b]) & (nan[a] | (np.asarray(vals[a] == vals[b], dtype=bool)))
        diff |= (va != vb) | (both & ~same)
    return diff


def _resorted(cols, n: int) -> np.ndarray:
    """The helper's stable re-sort under EXCLUDE with null keys: rows with a
    null key after the others (then cut off), the rest ascending by key
    column, NaN above every number."""
    seq = []
    for valid, vals, nan in reversed(cols):
        _, rank = np.unique(vals, return_inverse=True)
        seq.append(rank.reshape(-1))
        seq.append(nan.astype(np.int8))
    any_null = np.zeros(n, dtype=bool)
    for valid, _, _ in cols:
        any_null |= ~valid
    seq.append(any_null.astype(np.int8))
    order = np.lexsort(seq)  # stable
    return order[: int(n - any_null.sum())]


def sorted_groups(keys: Sequence[HostCol], null_policy) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(label per row, row kept, first row per group): label g for the rows of
    the g-th group in output order."""
    n = keys[0].size if keys else 0
    cols = [_key_rows(k) for k in keys]
    has_nulls = any(not c[0].all() for c in cols)
    if null_policy == NullPolicy.EXCLUDE and has_nulls:
        order = _resorted(cols, n)
    else:
        order = np.arange(n, dtype=np.int64)
    start = np.ones(len(order), dtype=bool)
    if len(order) > 1:
        start[1:] = _rows_differ(cols, order[1:], order[:-1])
    label = np.zeros(n, dtype=np.int32)
    kept = np.zeros(n, dtype=bool)
    label[order] = (np.cumsum(start) - 1).astype(np.int32)
    kept[order] = True
    return label, kept, order[start]


def _rows_of_groups(perm: np.ndarray, per: int) -> np.ndarray:
    if per == 1:
        return perm
    return (perm[:, None] * per + np.arange(per)[None, :]).reshape(-1)


def _key_at(k: HostCol, rows: np.ndarray, null_policy):
    """One output key column in oracle.groupby's (type_id, values, valid) form."""
    s = slice(k.offset, k.offset + k.size)
    valid = None
    if k.valid is not None and null_policy == NullPolicy.INCLUDE:
        valid = np.asarray(k.valid, dtype=bool)[s][rows]
    vals = k.values[s][rows]
    if k.type_id == TypeId.STRING:
        vals = np.array(["" if v is None else v for v in vals], dtype=object)
    elif k.type_id == TypeId.BOOL8:
        vals = vals.astype(bool)
    elif k.type_id == TypeId.DICTIONARY32:
        vals = vals.astype(np.int32)
    return int(k.type_id), vals, valid


def groupby(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, threads: int = 1) -> dict:
    """oracle.groupby's result for keys declared sorted, in the reference's
    group order; adds "label" (the label column the groups were aggregated
    by) and "perm" (the plain oracle's group order to output order)."""
    label, kept, first = sorted_groups(keys, null_policy)
    lcol = HostCol(label, None if kept.all() else kept)
    r = orc.groupby([lcol], requests, NullPolicy.EXCLUDE, threads)
    g = r["num_groups"]
    perm = np.argsort(np.asarray(r["keys"][0][1], dtype=np.int64), kind="stable")
    assert g == len(first), f"{g} groups for {len(first)} first rows"
    results: List[list] = []
    for cols in r["results"]:
        out = []
        for tid, vals, valid in cols:
            per = len(vals) // g if g else 1
            rows = _rows_of_groups(perm, max(per, 1)) if g else np.zeros(0, np.int64)
            out.append((tid, np.asarray(vals)[rows], None if valid is None else np.asarray(valid)[rows]))
        results.append(out)
    return {"num_groups": g, "keys": [_key_at(k, first, null_policy) for k in keys], "results": results,
            "label": lcol, "perm": perm}
