"""GPU parity of groupbys created with keys_are_sorted (sorted::YES) against
the sort-path oracle (oracle/presorted.py), through the C ABI: groups are the
runs of equal adjacent rows in row order (nulls equal, NaNs equal, -0.0 ==
0.0), or, under EXCLUDE with null keys, one group per key ordered by its first
row -- compared in output order, not sorted.  Tolerances are those of
tests/gbx_testing.py."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, Strategy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

QS = [0.0, 0.3, 0.5, 1.0]


def _aggs():
    return [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.COUNT_ALL, 0), (Kind.MIN, 0), (Kind.MAX, 0),
            (Kind.MEAN, 0), (Kind.VARIANCE, 1), (Kind.ARGMIN, 0), (Kind.ARGMAX, 0), (Kind.MEDIAN, 0),
            (Kind.QUANTILE, 0, {"quantiles": QS, "interpolation": 0}), (Kind.NUNIQUE, 0),
            (Kind.NTH_ELEMENT, 0, {"null_policy": NullPolicy.INCLUDE}), (Kind.M2, 0)]


def _sorted_keys(rng, n, card, dtype=np.int32, descending=False):
    k = np.sort(rng.integers(0, card, n)).astype(dtype)
    return k[::-1].copy() if descending else k


@pytest.mark.parametrize("descending", [False, True])
@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_sorted_keys_without_nulls(policy, descending):
    rng = np.random.default_rng(41)
    n = 200_000
    k = _sorted_keys(rng, n, 5_000, np.int64, descending)
    v = rng.normal(0, 10, n)
    w = rng.integers(-100, 100, n).astype(np.int32)
    wv = rng.random(n) >= 0.2
    T.assert_parity([HostCol(k)], [(HostCol(v), _aggs()), (HostCol(w, wv), _aggs())], policy,
                    keys_are_sorted=True)


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_sorted_keys_with_null_runs(policy):
    """INCLUDE: each run of null keys is a group of its own; EXCLUDE: the
    null rows drop out and each key is one group."""
    rng = np.random.default_rng(42)
    n = 150_000
    k = _sorted_keys(rng, n, 2_000)
    kv = np.ones(n, dtype=bool)
    for s in rng.integers(0, n - 50, 300):
        kv[s:s + rng.integers(1, 40)] = False
    v = rng.integers(-1000, 1000, n).astype(np.int64)
    T.assert_parity([HostCol(k, kv)], [(HostCol(v), _aggs())], policy, keys_are_sorted=True)


def test_keys_not_actually_sorted_split_into_runs():
    rng = np.random.default_rng(43)
    n = 100_000
    k = rng.integers(0, 4, n).astype(np.int16)  # many short runs of few keys
    v = rng.random(n).astype(np.float32)
    got, want = T.assert_parity([HostCol(k)], [(HostCol(v), [(Kind.SUM, 0), (Kind.COUNT_ALL, 0)])],
                                keys_are_sorted=True)
    assert got["num_groups"] > 4 * 1000


def test_float_keys_nan_and_signed_zero_runs():
    n = 64_000
    rng = np.random.default_rng(44)
    f = np.sort(rng.integers(-5, 5, n).astype(np.float64))
    f[f == 0] = np.where(rng.random(int((f == 0).sum())) < 0.5, -0.0, 0.0)
    f[-3000:] = np.nan
    v = rng.integers(0, 9, n).astype(np.int32)
    T.assert_parity([HostCol(f)], [(HostCol(v), [(Kind.SUM, 0), (Kind.ARGMAX, 0)])], keys_are_sorted=True)


def test_string_and_multicolumn_keys():
    rng = np.random.default_rng(45)
    n = 40_000
    words = np.array(sorted(["", "a", "ab", "abc", "b", "año", "₹1", "zz", "z" * 40]), dtype=object)
    s = words[np.sort(rng.integers(0, len(words), n))]
    sv = rng.random(n) >= 0.05
    d = rng.integers(0, 3, n).astype(np.int8)
    t = rng.integers(0, 1 << 40, n).astype(np.int64)
    keys = [HostCol(list(s), sv, type_id=TypeId.STRING), HostCol(d)]
    v = rng.normal(0, 1, n)
    T.assert_parity(keys, [(HostCol(v), [(Kind.SUM, 0), (Kind.MEDIAN, 0), (Kind.COUNT_ALL, 0)])],
                    NullPolicy.INCLUDE, keys_are_sorted=True)
    # three wide columns (beyond 128 packed bits)
    keys = [HostCol(np.sort(t)), HostCol(t), HostCol(t ^ 7)]
    T.assert_parity(keys, [(HostCol(v), [(Kind.MAX, 0)])], keys_are_sorted=True)


@pytest.mark.parametrize("strategy", [Strategy.AUTO, Strategy.PRIVATIZED, Strategy.GLOBAL, Strategy.WARP,
                                      Strategy.PARTITIONED, Strategy.BUCKETED], ids=lambda s: s.name)
def test_every_strategy_on_the_labels(strategy):
    rng = np.random.default_rng(46)
    n = 300_000
    k = _sorted_keys(rng, n, 100_000)
    v = rng.integers(-50, 50, n).astype(np.int32)
    T.assert_parity([HostCol(k)], [(HostCol(v), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.ARGMIN, 0), (Kind.MEAN, 0)])],
                    strategy=strategy, keys_are_sorted=True)


def test_many_rows():
    rng = np.random.default_rng(47)
    n = 3_000_000
    k = _sorted_keys(rng, n, 400_000)
    v = rng.integers(-(1 << 30), 1 << 30, n).astype(np.int64)
    T.assert_parity([HostCol(k)], [(HostCol(v), [(Kind.SUM, 0), (Kind.NUNIQUE, 0), (Kind.MAX, 0)])],
                    keys_are_sorted=True, threads=8)


def test_empty_all_null_and_sliced():
    e = np.zeros(0, np.int32)
    T.assert_parity([HostCol(e)], [(HostCol(np.zeros(0)), [(Kind.SUM, 0)])], keys_are_sorted=True)
    k = np.array([1, 1, 2, 2, 3], np.int32)
    v = np.arange(5.0)
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([HostCol(k, np.zeros(5, bool))], [(HostCol(v), [(Kind.SUM, 0), (Kind.COUNT_ALL, 0)])],
                        policy, keys_are_sorted=True)
    ks = HostCol(np.array([7, 1, 1, 2, 2, 2, 7], np.int32), offset=1, size=5)
    vs = HostCol(np.arange(7, dtype=np.int32), offset=1, size=5)
    T.assert_parity([ks], [(vs, [(Kind.SUM, 0), (Kind.ARGMIN, 0)])], keys_are_sorted=True)


def test_reference_nulls_before_include_nulls():
    """keys_tests.cpp:199-225: two null runs are two groups, in row order."""
    k = HostCol(np.array([1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4], np.int32),
                np.array([1, 1, 1, 0, 0, 1, 1, 0, 1, 1, 1], bool))
    v = HostCol(np.arange(11, dtype=np.int32) % 10 + np.array([0] * 10 + [4], np.int32))
    got = T.run_gpu([k], [(v, [(Kind.SUM, 0)])], NullPolicy.INCLUDE, keys_are_sorted=True)
    assert list(got["keys"][0][2]) == [True, False, True, False, True, True]
    assert list(got["keys"][0][1][[0, 2, 4, 5]]) == [1, 2, 3, 4]
    assert list(got["results"][0][0][1]) == [3, 7, 11, 7, 17, 4]
