"""Groupby over STRUCT key columns, restated on top of the plain oracle.

TEST INFRASTRUCTURE ONLY: the parity checker for libgbx's STRUCT keys
(tests/).  Nothing in the product imports it.

The reference compares struct keys with its nested row comparator
(table/experimental/row_operators.cuh:1456-1500, used by the hash groupby's
set, groupby/hash/groupby.cu:555-566): two struct rows are equal when both
are null, or both are valid and every member is equal (recursively; nulls
equal, NaNs equal, -0.0 == +0.0).  So a valid struct whose members are all
null is not the null struct (structs_tests.cpp:179-211).  Rows with a null
key are dropped under EXCLUDE by the AND of the key columns' own masks
(hash/groupby.cu:560-567): a null member of a valid struct does not drop the
row.  A key's output is gathered from its representative row, and a gathered
struct's members carry the struct's nulls.

Restated by flattening: each key column becomes leaves -- a STRUCT its own
validity, then its members' leaves; any other column itself -- with each
leaf's validity its own AND every enclosing struct's.  Two rows are equal when
every leaf is (validity, then value where valid).  The plain oracle
(oracle.groupby) groups the rows by those leaves encoded without nulls (a
validity indicator and the value with nulls read as 0 or ""), after a first
column that is null where a key column itself is null, under EXCLUDE.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from cudf_b200._abi import NullPolicy, TypeId
from oracle import oracle as orc
from oracle.oracle import HostCol


@dataclass
class Leaf:
    type_id: int
    values: Optional[np.ndarray]  # None for a struct's validity leaf
    valid: np.ndarray             # its own validity AND every enclosing struct's
    own: np.ndarray               # its own validity


def leaves(col: HostCol, n: int, base: int = 0, enclosing: Optional[np.ndarray] = None) -> List[Leaf]:
    """The leaves of rows [0, n) of a column whose row r is element
    base + col.offset + r."""
    lo = base + col.offset
    own = np.ones(n, dtype=bool) if col.valid is None else np.asarray(col.valid, dtype=bool)[lo:lo + n]
    eff = own if enclosing is None else own & enclosing
    if col.type_id == TypeId.STRUCT:
        out = [Leaf(int(TypeId.STRUCT), None, eff, own)]
        for m in col.children:
            out += leaves(m, n, lo, eff)
        return out
    vals = col.values[lo:lo + n]
    if col.type_id == TypeId.STRING:
        vals = np.array(["" if v is None else v for v in vals], dtype=object)
    return [Leaf(int(col.type_id), vals, eff, own)]


def _encoded(leaf: Leaf, src: HostCol) -> List[HostCol]:
    """A leaf as columns without nulls: its validity, and its value (0 / ""
    where null)."""
    out = [HostCol(leaf.valid.astype(np.uint8))]
    if leaf.values is None:
        return out
    if leaf.type_id == TypeId.STRING:
        out.append(HostCol([v if ok else "" for v, ok in zip(leaf.values, leaf.valid)], type_id=TypeId.STRING))
    elif leaf.type_id == TypeId.DICTIONARY32:
        out.append(HostCol(np.where(leaf.valid, leaf.values, 0).astype(np.int64)))
    else:
        v = np.asarray(leaf.values)
        out.append(HostCol(np.where(leaf.valid, v, np.zeros(1, dtype=v.dtype)).astype(v.dtype), type_id=leaf.type_id,
                           scale=src.scale))
    return out


def _leaf_sources(col: HostCol) -> List[HostCol]:
    """The column behind each leaf (for scales), in leaf order."""
    if col.type_id != TypeId.STRUCT:
        return [col]
    out = [col]
    for m in col.children:
        out += _leaf_sources(m)
    return out


def groupby(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, threads: int = 1) -> dict:
    """oracle.groupby's result with the key columns flattened to leaves:
    "keys" holds one (type_id, values, valid) per leaf (a struct's validity
    leaf with type STRUCT and no values), valid being the leaf's validity in
    the output (its own AND its enclosing structs'); "enc" is the null-free
    key table the plain oracle grouped by (same group order)."""
    n = keys[0].size if keys else 0
    lv: List[Leaf] = []
    src: List[HostCol] = []
    top_null = np.zeros(n, dtype=bool)
    for k in keys:
        ls = leaves(k, n)
        top_null |= ~ls[0].own
        lv += ls
        src += _leaf_sources(k)
    enc: List[HostCol] = []
    if null_policy == NullPolicy.EXCLUDE and top_null.any():
        enc.append(HostCol(np.zeros(n, dtype=np.int8), ~top_null))
    spans = []
    for leaf, s in zip(lv, src):
        e = _encoded(leaf, s)
        spans.append((len(enc), len(e)))
        enc += e
    r = orc.groupby(enc, requests, NullPolicy.EXCLUDE, threads)
    g = r["num_groups"]
    out_keys = []
    for leaf, (at, cnt) in zip(lv, spans):
        valid = np.asarray(r["keys"][at][1]).astype(bool)
        if cnt == 1:
            out_keys.append((int(TypeId.STRUCT), np.zeros(g, dtype=bool), valid))
        else:
            tid, vals, _ = r["keys"][at + 1]
            if leaf.type_id == TypeId.DICTIONARY32:
                vals = np.asarray(vals).astype(np.int32)
            out_keys.append((int(leaf.type_id), vals, valid))
    return {"num_groups": g, "keys": out_keys, "results": r["results"], "enc": enc}


def _rows(type_id: int, values, valid) -> int:
    if valid is not None:
        return len(valid)
    if type_id == TypeId.STRUCT:
        return _rows(*values[0]) if values else 0
    return len(values)


def flatten_output(type_id: int, values, valid, enclosing: Optional[np.ndarray] = None) -> list:
    """An output key column -- (type_id, values, valid), a STRUCT column's
    values being its members' (type_id, values, valid) -- as the leaves
    groupby() lists."""
    if type_id == TypeId.STRUCT:
        members = values
        n = _rows(type_id, values, valid)
        own = np.ones(n, dtype=bool) if valid is None else np.asarray(valid, dtype=bool)
        eff = own if enclosing is None else own & enclosing
        out = [(int(TypeId.STRUCT), np.zeros(n, dtype=bool), eff)]
        for (mt, mv, mvalid) in members:
            out += flatten_output(mt, mv, mvalid, eff)
        return out
    vals = np.asarray(values) if type_id != TypeId.STRING else values
    m = len(vals)
    own = np.ones(m, dtype=bool) if valid is None else np.asarray(valid, dtype=bool)
    eff = own if enclosing is None else own & enclosing
    return [(int(type_id), vals, eff)]
