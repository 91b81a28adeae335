"""The sorted::YES oracle (oracle/presorted.py) against a row-by-row
restatement of the reference's sort-path grouping
(groupby/sort/sort_helper.cu:64-71, 96-104, 141-179): runs of equal adjacent
rows (nulls equal, NaNs equal, -0.0 == 0.0) in row order, or, under EXCLUDE
with null keys, one group per key in ascending key order."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle import oracle as orc
from oracle import presorted as P
from oracle.oracle import HostCol


def _cell(k: HostCol, r: int):
    """A comparable cell: None for null, NaN folded to one marker."""
    if k.valid is not None and not k.valid[r]:
        return None
    v = k.values[r]
    if k.type_id == TypeId.STRING:
        return v
    if isinstance(v, (float, np.floating)) and math.isnan(v):
        return ("nan",)
    return float(v) if isinstance(v, (float, np.floating)) else int(v)


def _brute_runs(keys, values, valid):
    """[(key tuple, sum of valid values, first row)] per run."""
    n = keys[0].size
    out = []
    for r in range(n):
        key = tuple(_cell(k, r) for k in keys)
        x = int(values[r]) if valid is None or valid[r] else 0
        if out and out[-1][0] == key:
            out[-1][1] += x
        else:
            out.append([key, x, r])
    return out


def _sum_result(res):
    return [int(v) if ok else 0 for v, ok in zip(res["results"][0][0][1], res["results"][0][0][2]
                                                  if res["results"][0][0][2] is not None
                                                  else [True] * res["num_groups"])]


@pytest.mark.parametrize("policy", [NullPolicy.INCLUDE, NullPolicy.EXCLUDE], ids=lambda p: p.name)
@pytest.mark.parametrize("seed", range(6))
def test_runs_match_row_by_row(policy, seed):
    rng = np.random.default_rng(seed)
    n = 300
    a = np.sort(rng.integers(0, 12, n)).astype(np.int32)
    b = rng.integers(0, 2, n).astype(np.float64)
    b[rng.random(n) < 0.1] = np.nan
    b[rng.random(n) < 0.1] = -0.0
    av = rng.random(n) >= 0.1 if policy == NullPolicy.INCLUDE else None
    keys = [HostCol(a, av), HostCol(b)]
    v = rng.integers(-5, 5, n).astype(np.int64)
    res = P.groupby(keys, [(HostCol(v), [(Kind.SUM, 0)])], policy)
    runs = _brute_runs(keys, v, None)
    assert res["num_groups"] == len(runs)
    assert _sum_result(res) == [r[1] for r in runs]
    first = [r[2] for r in runs]
    assert np.array_equal(res["keys"][0][1], a[first])


def test_unsorted_rows_split_equal_keys():
    """Equal keys that are not adjacent form separate groups."""
    k = HostCol(np.array([1, 1, 2, 1, 1, 3, 2], np.int32))
    v = HostCol(np.arange(7, dtype=np.int32))
    res = P.groupby([k], [(v, [(Kind.SUM, 0), (Kind.COUNT_ALL, 0)])])
    assert list(res["keys"][0][1]) == [1, 2, 1, 3, 2]
    assert list(res["results"][0][0][1]) == [1, 2, 7, 5, 6]
    assert list(res["results"][0][1][1]) == [2, 1, 2, 1, 1]


def test_exclude_with_null_keys_sorts_again():
    """EXCLUDE with null keys: one group per key, ascending, nulls dropped,
    whatever the row order (sort_helper.cu:64-71)."""
    rng = np.random.default_rng(3)
    n = 400
    k = rng.integers(-20, 20, n).astype(np.int64)
    kv = rng.random(n) >= 0.2
    v = rng.integers(0, 100, n).astype(np.int32)
    res = P.groupby([HostCol(k, kv)], [(HostCol(v), [(Kind.SUM, 0)])], NullPolicy.EXCLUDE)
    plain = orc.groupby([HostCol(k, kv)], [(HostCol(v), [(Kind.SUM, 0)])], NullPolicy.EXCLUDE)
    got_keys = res["keys"][0][1]
    assert np.all(np.diff(got_keys) > 0)
    o = np.argsort(plain["keys"][0][1])
    assert np.array_equal(got_keys, plain["keys"][0][1][o])
    assert np.array_equal(res["results"][0][0][1], plain["results"][0][0][1][o])


def test_string_runs_and_nan_runs():
    s = HostCol(["a", "a", None, None, "b", "a", ""], type_id=TypeId.STRING)
    f = np.array([np.nan, np.nan, 0.0, -0.0, 1.0, 1.0, 1.0])
    v = HostCol(np.ones(7, np.int32))
    res = P.groupby([s, HostCol(f)], [(v, [(Kind.COUNT_ALL, 0)])], NullPolicy.INCLUDE)
    # runs: (a,nan)x2, (null,0)x2, (b,1), (a,1), ("",1)
    assert list(res["results"][0][0][1]) == [2, 2, 1, 1, 1]
    assert list(res["keys"][0][2]) == [True, False, True, True, True]


def test_quantile_columns_follow_group_order():
    k = HostCol(np.array([5, 5, 5, 2, 2, 9], np.int32))
    v = HostCol(np.array([1.0, 2.0, 3.0, 10.0, 20.0, 7.0]))
    res = P.groupby([k], [(v, [(Kind.QUANTILE, 0, {"quantiles": [0.0, 1.0], "interpolation": 0})])])
    assert list(res["keys"][0][1]) == [5, 2, 9]
    assert list(res["results"][0][0][1]) == [1.0, 3.0, 10.0, 20.0, 7.0, 7.0]


def test_empty_and_sliced_keys():
    res = P.groupby([HostCol(np.zeros(0, np.int32))], [(HostCol(np.zeros(0)), [(Kind.SUM, 0)])])
    assert res["num_groups"] == 0
    k = HostCol(np.array([9, 1, 1, 2, 2, 9], np.int32), offset=1, size=4)
    v = HostCol(np.array([100, 1, 2, 3, 4, 100], np.int32), offset=1, size=4)
    res = P.groupby([k], [(v, [(Kind.SUM, 0)])])
    assert list(res["keys"][0][1]) == [1, 2] and list(res["results"][0][0][1]) == [3, 7]
