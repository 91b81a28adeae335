"""CPU tests of distinct rows and the distinct-key join: the oracle
(oracle/distinct.py) against the reference gtests' known answers and against
pandas, and the C ABI's argument checks and empty inputs (no device work)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pandas as pd
import pytest

from cudf_b200 import _abi, _lib
from cudf_b200._abi import TypeId
from oracle import distinct as od
from tests.golden import distinct_kats as K


def host_cols(spec):
    return [(np.array(v, dtype=t), None if m is None else np.array(m, bool)) for v, m, t in spec]


@pytest.mark.parametrize("case", K.DISTINCT_COUNT, ids=[c[0] for c in K.DISTINCT_COUNT])
def test_oracle_distinct_count_kat(case):
    _, spec, eq, uneq = case
    cols = host_cols(spec)
    assert od.distinct_count(cols, True) == eq
    assert od.distinct_count(cols, False) == uneq


def test_oracle_distinct_count_table_no_null():
    a, b = K.TABLE_NO_NULL
    want = len(set(zip(a, b)))
    assert od.distinct_count([(np.array(a), None), (np.array(b), None)]) == want


@pytest.mark.parametrize("case", K.DISTINCT, ids=[c[0] for c in K.DISTINCT])
def test_oracle_distinct_indices_kat(case):
    _, spec, ne, nan_eq, want = case
    cols = host_cols(spec)
    for keep, rows in want.items():
        assert list(od.distinct_indices(cols, keep, ne, nan_eq)) == rows, keep


def test_oracle_any_with_nans_kat():
    spec, want = K.ANY_WITH_NANS
    cols = host_cols(spec)
    for nan_eq, n in want.items():
        assert len(od.distinct_indices(cols, 0, True, nan_eq)) == n


@pytest.mark.parametrize("case", K.JOIN, ids=[c[0] for c in K.JOIN])
def test_oracle_join_kat(case):
    _, b, p, ne, inner, left = case
    bc, pc = host_cols(b), host_cols(p)
    if inner is not None:
        assert [tuple(x) for x in od.distinct_join(bc, pc, ne)] == inner
    if left is not None:
        got = od.distinct_join(bc, pc, ne, left=True)
        assert [None if x == -(2 ** 31) else int(x) for x in got] == left


def test_oracle_matches_pandas():
    rng = np.random.default_rng(1)
    n = 3000
    a = rng.integers(0, 30, n)
    b = rng.choice([0.5, 1.5, -0.0, 0.0, np.nan], n)
    cols = [(a, None), (b, None)]
    df = pd.DataFrame({"a": a, "b": np.where(b == 0, 0.0, b)})
    assert od.distinct_count(cols) == len(df.drop_duplicates())
    first = od.distinct_indices(cols, 1)
    assert list(first) == list(np.sort(df.drop_duplicates(keep="first").index.to_numpy()))
    last = od.distinct_indices(cols, 2)
    assert list(last) == list(np.sort(df.drop_duplicates(keep="last").index.to_numpy()))
    none = od.distinct_indices(cols, 3)
    assert list(none) == list(np.sort(df.drop_duplicates(keep=False).index.to_numpy()))
    # join against a merge on a distinct build side
    bdf = df.drop_duplicates().reset_index().rename(columns={"index": "bi"})
    probe = pd.DataFrame({"a": rng.integers(0, 40, 500), "b": rng.choice([0.5, 1.5, 0.0, np.nan], 500)})
    m = probe.reset_index().rename(columns={"index": "pi"}).merge(bdf, on=["a", "b"], how="inner")
    want = sorted(zip(m.bi, m.pi))
    got = od.distinct_join([(bdf.a.to_numpy(), None), (bdf.b.to_numpy(), None)],
                           [(probe.a.to_numpy(), None), (probe.b.to_numpy(), None)])
    assert [tuple(x) for x in got] == [(int(bdf.bi.tolist().index(bb)), int(pp)) for bb, pp in want]


def _tv(cols):
    arr = (_abi.gbx_column_view * max(1, len(cols)))()
    keep = []
    for i, (vals, tid) in enumerate(cols):
        arr[i].type_id = int(tid)
        arr[i].size = len(vals)
        keep.append(vals)
        arr[i].data = vals.ctypes.data if len(vals) else None
    tv = _abi.gbx_table_view(len(cols), 0, C.cast(arr, C.POINTER(_abi.gbx_column_view)))
    return tv, (arr, keep)


def test_abi_checks_before_device_work():
    lib = _lib.lib()
    a = np.arange(4, dtype=np.int32)
    b = np.arange(3, dtype=np.int32)
    tv, keep = _tv([(a, TypeId.INT32), (b, TypeId.INT32)])
    out = C.c_int64()
    assert lib.gbx_distinct_count(C.byref(tv), 0, None, None, C.byref(out)) == _abi.Status.ERR_LOGIC
    assert b"differ in size" in lib.gbx_last_error()
    tv1, keep1 = _tv([(a, TypeId.INT32)])
    col = _abi.gbx_column()
    assert lib.gbx_distinct_indices(C.byref(tv1), 7, 0, 0, None, None, C.byref(col)) == _abi.Status.ERR_LOGIC
    assert b"duplicate_keep_option" in lib.gbx_last_error()
    tvf, keepf = _tv([(np.arange(4, dtype=np.float32), TypeId.FLOAT32)])
    b1, b2 = _abi.gbx_column(), _abi.gbx_column()
    assert lib.gbx_distinct_join(C.byref(tv1), C.byref(tvf), 0, 0, None, None, C.byref(b1),
                                 C.byref(b2)) == _abi.Status.ERR_LOGIC
    assert b"data types" in lib.gbx_last_error()
    # a STRING key needs its offsets; list keys are not taken
    tvs, keeps = _tv([(a, TypeId.STRING)])
    assert lib.gbx_distinct_count(C.byref(tvs), 0, None, None, C.byref(out)) == _abi.Status.ERR_LOGIC
    assert b"offsets" in lib.gbx_last_error()
    tvl, keepl = _tv([(a, TypeId.LIST)])
    assert lib.gbx_distinct_count(C.byref(tvl), 0, None, None, C.byref(out)) == _abi.Status.ERR_UNSUPPORTED


def test_abi_empty_input_needs_no_device():
    lib = _lib.lib()
    e = np.zeros(0, dtype=np.int32)
    tv, keep = _tv([(e, TypeId.INT32)])
    out = C.c_int64(5)
    assert lib.gbx_distinct_count(C.byref(tv), 0, None, None, C.byref(out)) == 0
    assert out.value == 0
