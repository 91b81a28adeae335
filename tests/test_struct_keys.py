"""STRUCT keys on the CPU: the struct-key oracle (oracle/structs.py) against
the reference gtests' known answers (tests/golden/struct_kats.py), compared
leaf by leaf after sorting by key as the reference harness does
(groupby_test_util.cpp:89-96); plus the C-ABI checks of STRUCT key columns
that need no GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cudf_b200 import _abi
from cudf_b200._abi import Kind, NullPolicy, TypeId
from cudf_b200.column import storage_dtype
from oracle import structs as S
from oracle.oracle import HostCol
from tests import gbx_testing as T
from tests.golden import struct_kats as KAT

CASES = KAT.cases()


def host_of(spec) -> HostCol:
    kind = spec[0]
    if kind == "struct":
        _, members, valid = spec
        return HostCol(None, None if valid is None else np.array(valid, bool), type_id=TypeId.STRUCT,
                       children=[host_of(m) for m in members])
    if kind == "string":
        _, vals, valid = spec
        return HostCol(list(vals), None if valid is None else np.array(valid, bool), type_id=TypeId.STRING)
    _, t, vals, valid = spec
    arr = [0 if v is None else v for v in vals]
    if t == TypeId.BOOL8:
        a = np.array([bool(v) for v in arr], dtype=np.uint8)
    else:
        a = np.array(arr, dtype=storage_dtype(t)) if arr else np.zeros(0, storage_dtype(t))
    return HostCol(a, None if valid is None else np.array(valid, bool), type_id=t)


def typed_of(spec):
    """The spec as an output key column (type_id, values, valid)."""
    kind = spec[0]
    if kind == "struct":
        _, members, valid = spec
        return (int(TypeId.STRUCT), [typed_of(m) for m in members], None if valid is None else np.array(valid, bool))
    if kind == "string":
        _, vals, valid = spec
        return (int(TypeId.STRING), np.array(["" if v is None else v for v in vals], dtype=object),
                None if valid is None else np.array(valid, bool))
    _, t, vals, valid = spec
    arr = [0 if v is None else v for v in vals]
    if t == TypeId.BOOL8:
        a = np.array([bool(v) for v in arr], dtype=bool)
    else:
        a = np.array(arr, dtype=storage_dtype(t)) if arr else np.zeros(0, storage_dtype(t))
    return (int(t), a, None if valid is None else np.array(valid, bool))


def build(case):
    keys = [host_of(case["keys"])]
    vals = HostCol(np.array(case["values"], dtype=np.int32) if case["values"] else np.zeros(0, np.int32))
    return keys, [(vals, [(Kind.SUM, 0)])]


def check(got_leaves, got_sum, case):
    want_leaves = S.flatten_output(*typed_of(case["expect_keys"]))
    assert len(got_leaves) == len(want_leaves)
    n = len(case["expect"])
    assert len(got_sum[1]) == n, f"{len(got_sum[1])} groups, expected {n}"
    go = T.sort_order(got_leaves)
    wo = T.sort_order(want_leaves)
    T.compare_keys(got_leaves, want_leaves, go, wo)
    want_sum = (int(TypeId.INT64), np.array(case["expect"], dtype=np.int64) if n else np.zeros(0, np.int64), None)
    T.compare_values(Kind.SUM, got_sum, want_sum, go, wo, ctx=case["id"])


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_matches_struct_kat(case):
    keys, reqs = build(case)
    r = S.groupby(keys, reqs, NullPolicy.INCLUDE)
    check(r["keys"], r["results"][0][0], case)


def test_exclude_drops_null_structs_not_null_members():
    """EXCLUDE drops rows whose struct is null, keeps rows whose member is."""
    m0 = HostCol(np.array([1, 1, 2, 2], np.int32), np.array([1, 0, 1, 1], bool))
    k = HostCol(None, np.array([1, 1, 1, 0], bool), type_id=TypeId.STRUCT, children=[m0])
    v = HostCol(np.array([1, 2, 3, 4], np.int32))
    r = S.groupby([k], [(v, [(Kind.SUM, 0)])], NullPolicy.EXCLUDE)
    assert r["num_groups"] == 3
    assert sorted(int(x) for x in r["results"][0][0][1]) == [1, 2, 3]


def _lib():
    from cudf_b200 import _lib as L
    return L.lib()


def test_struct_key_views_are_checked_at_create():
    """A STRUCT key column needs its members; members must cover its rows;
    dictionary and list members are refused."""
    lib = _lib()
    a = np.arange(4, dtype=np.int32)
    m = _abi.gbx_column_view()
    m.type_id = int(TypeId.INT32)
    m.size = 4
    m.data = a.ctypes.data
    members = (_abi.gbx_column_view * 1)(m)
    sv = _abi.gbx_column_view()
    sv.type_id = int(TypeId.STRUCT)
    sv.size = 4
    sv.num_children = 1
    sv.dict_keys = C.cast(members, C.POINTER(_abi.gbx_column_view))
    tv = _abi.gbx_table_view()
    tv.num_columns = 1
    tv.columns = C.pointer(sv)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.OK
    lib.gbx_groupby_destroy(h)
    sv.num_children = 0
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.ERR_LOGIC
    sv.num_children = 1
    sv.offset = 1  # rows 1..4 of a 4-row member
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.ERR_LOGIC
    sv.offset = 0
    members[0].type_id = int(TypeId.LIST)
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.ERR_UNSUPPORTED
