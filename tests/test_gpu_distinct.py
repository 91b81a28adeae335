"""GPU parity of distinct_count / distinct_indices / distinct and the
distinct-key inner and left joins (through the C ABI) with the oracle
(oracle/distinct.py): the reference gtests' known answers, then seeded inputs
with nulls, NaNs, signed zeros, composite keys and every keep option, at
sizes from a few rows to millions."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200 import Column, Table
from cudf_b200 import stream_compaction as sc
from cudf_b200._abi import DuplicateKeep, NanEquality, NullEquality, TypeId
from oracle import distinct as od
from tests.golden import distinct_kats as K

pytestmark = pytest.mark.gpu


def dev_table(spec):
    cols = []
    for v, m, t in spec:
        vals = np.array(v, dtype=t)
        cols.append(Column.from_numpy(vals, None if m is None else np.array(m, bool)))
    return Table(cols)


def host_cols(spec):
    return [(np.array(v, dtype=t), None if m is None else np.array(m, bool)) for v, m, t in spec]


def ne(b):
    return NullEquality.EQUAL if b else NullEquality.UNEQUAL


def nan_eq(b):
    return NanEquality.ALL_EQUAL if b else NanEquality.UNEQUAL


@pytest.mark.parametrize("case", K.DISTINCT_COUNT, ids=[c[0] for c in K.DISTINCT_COUNT])
def test_distinct_count_kat(case):
    cid, spec, eq, uneq = case
    t = dev_table(spec)
    assert sc.distinct_count(t, NullEquality.EQUAL) == eq
    assert sc.distinct_count(t, NullEquality.UNEQUAL) == uneq


@pytest.mark.parametrize("case", K.DISTINCT, ids=[c[0] for c in K.DISTINCT])
def test_distinct_indices_kat(case):
    _, spec, nulls, nans, want = case
    t = dev_table(spec)
    for keep, rows in want.items():
        got = np.sort(sc.distinct_indices(t, DuplicateKeep(keep), ne(nulls), nan_eq(nans)).to_numpy()[0])
        assert list(got) == rows, keep


def test_keep_any_with_nans_kat():
    spec, want = K.ANY_WITH_NANS
    t = dev_table(spec)
    for nans, n in want.items():
        assert len(sc.distinct_indices(t, DuplicateKeep.KEEP_ANY, NullEquality.EQUAL, nan_eq(nans))) == n


@pytest.mark.parametrize("case", K.JOIN, ids=[c[0] for c in K.JOIN])
def test_join_kat(case):
    _, b, p, nulls, inner, left = case
    bt, pt = dev_table(b), dev_table(p)
    if inner is not None:
        bi, pi = sc.distinct_inner_join(bt, pt, ne(nulls))
        got = sorted(zip(bi.to_numpy()[0].tolist(), pi.to_numpy()[0].tolist()))
        assert got == inner
    if left is not None:
        got = sc.distinct_left_join(bt, pt, ne(nulls)).to_numpy()[0]
        assert [None if x == sc.JOIN_NONE else int(x) for x in got] == left


def test_integer_inner_join_kat():
    """distinct_join_tests.cpp:84 IntegerInnerJoin: build 0..2023, probe 0, 2, ..."""
    size = 2024
    bt = Table([Column.from_numpy(np.arange(size, dtype=np.int32))])
    pt = Table([Column.from_numpy(np.arange(0, 2 * size, 2, dtype=np.int32))])
    bi, pi = sc.distinct_inner_join(bt, pt)
    b = bi.to_numpy()[0]
    p = pi.to_numpy()[0]
    assert len(b) == size // 2
    assert np.array_equal(np.sort(b), np.arange(0, size, 2))
    assert np.array_equal(b, 2 * p)


def _random_keys(rng, n, card, kind):
    if kind == "int64":
        return [(rng.integers(0, card, n).astype(np.int64), None)]
    if kind == "int32_nulls":
        return [(rng.integers(0, card, n).astype(np.int32), rng.random(n) >= 0.1)]
    if kind == "float_nan_zero":
        v = rng.integers(0, card, n).astype(np.float64) - card / 2
        v[rng.random(n) < 0.05] = np.nan
        v[rng.random(n) < 0.05] = -0.0
        return [(v, rng.random(n) >= 0.05)]
    # composite (int32 nullable, int16)
    return [(rng.integers(0, card, n).astype(np.int32), rng.random(n) >= 0.05),
            (rng.integers(-3, 3, n).astype(np.int16), None)]


def _dev(cols):
    return Table([Column.from_numpy(v, m) for v, m in cols])


@pytest.mark.parametrize("kind", ["int64", "int32_nulls", "float_nan_zero", "composite"])
@pytest.mark.parametrize("n,card", [(5_000, 50), (200_000, 20_000), (2_000_000, 300)])
def test_distinct_parity(kind, n, card):
    rng = np.random.default_rng(n + card)
    cols = _random_keys(rng, n, card, kind)
    t = _dev(cols)
    for nulls in (True, False):
        assert sc.distinct_count(t, ne(nulls)) == od.distinct_count(cols, nulls)
    if n > 200_000:
        return  # the oracle's per-row Python keys: counts only at this size
    for nulls in (True, False):
        for nans in (True, False):
            for keep in (1, 2, 3):
                got = np.sort(sc.distinct_indices(t, DuplicateKeep(keep), ne(nulls), nan_eq(nans)).to_numpy()[0])
                want = od.distinct_indices(cols, keep, nulls, nans)
                assert np.array_equal(got, want), (nulls, nans, keep)
            anyk = sc.distinct_indices(t, DuplicateKeep.KEEP_ANY, ne(nulls), nan_eq(nans)).to_numpy()[0]
            assert len(anyk) == len(od.distinct_indices(cols, 0, nulls, nans))


@pytest.mark.parametrize("kind", ["int64", "int32_nulls", "float_nan_zero", "composite"])
def test_join_parity(kind):
    rng = np.random.default_rng(7)
    build = _random_keys(rng, 20_000, 40_000, kind)
    # a distinct build side: first occurrences only
    keep = od.distinct_indices(build, 1, True, True)
    build = [(v[keep], None if m is None else m[keep]) for v, m in build]
    probe = _random_keys(rng, 50_000, 40_000, kind)
    bt, pt = _dev(build), _dev(probe)
    for nulls in (True, False):
        bi, pi = sc.distinct_inner_join(bt, pt, ne(nulls))
        got = sorted(zip(bi.to_numpy()[0].tolist(), pi.to_numpy()[0].tolist()))
        want = [tuple(x) for x in od.distinct_join(build, probe, nulls).tolist()]
        assert got == want, nulls
        left = sc.distinct_left_join(bt, pt, ne(nulls)).to_numpy()[0]
        assert np.array_equal(left, od.distinct_join(build, probe, nulls, left=True)), nulls


def test_distinct_table_gathers_rows():
    t = Table([Column.from_numpy(np.array([5, 5, 7, 5, 7], np.int64)),
               Column.from_numpy(np.array([1.0, 2.0, 3.0, 4.0, 5.0]))])
    out = sc.distinct(t, [0], DuplicateKeep.KEEP_LAST)
    k, v = out[0].to_numpy()[0], out[1].to_numpy()[0]
    order = np.argsort(k)
    assert list(k[order]) == [5, 7] and list(v[order]) == [4.0, 5.0]
