"""GPU parity of the sort-path kinds (M2, MEDIAN, QUANTILE, NUNIQUE,
NTH_ELEMENT) against the oracle, through the C ABI, on seeded inputs: value
types, nulls in keys and values, NaN and signed zeros, dictionary values,
two-word keys, every strategy, several requests on one column and sizes that
take many radix tiles.  Tolerances are those of tests/gbx_testing.py (MEDIAN /
QUANTILE equal to the oracle; NUNIQUE / NTH_ELEMENT bit-exact)."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, Strategy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

STRATS = [Strategy.AUTO, Strategy.PRIVATIZED, Strategy.GLOBAL, Strategy.WARP, Strategy.PARTITIONED,
          Strategy.BUCKETED]
QS = [0.0, 0.1, 0.25, 0.5, 0.77, 0.9, 1.0]


def sorted_aggs(numeric=True):
    """Every sorted kind with its options; MEDIAN / QUANTILE / M2 only over
    arithmetic values."""
    aggs = [(Kind.NUNIQUE, 0, {"null_policy": NullPolicy.EXCLUDE}),
            (Kind.NUNIQUE, 0, {"null_policy": NullPolicy.INCLUDE}),
            (Kind.NTH_ELEMENT, 0, {"null_policy": NullPolicy.INCLUDE}),
            (Kind.NTH_ELEMENT, -1, {"null_policy": NullPolicy.EXCLUDE}),
            (Kind.NTH_ELEMENT, 3, {"null_policy": NullPolicy.EXCLUDE})]
    if numeric:
        aggs = [(Kind.MEDIAN, 0), (Kind.M2, 0)] + [
            (Kind.QUANTILE, 0, {"quantiles": QS, "interpolation": i}) for i in range(5)] + aggs
    return aggs


def _values(dtype, n, rng):
    dt = np.dtype(dtype)
    if dt.kind == "f":
        v = (rng.normal(0, 50, n)).astype(dt)
        v[rng.random(n) < 0.01] = np.nan
        v[rng.random(n) < 0.01] = -0.0
        v[rng.random(n) < 0.01] = 0.0
        return v
    if dt.kind == "b":
        return rng.random(n) < 0.5
    info = np.iinfo(dt)
    return rng.integers(max(info.min, -1000), min(info.max, 1000), n, endpoint=True).astype(dt)


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint32, np.uint64,
                                   np.float32, np.float64, np.bool_])
def test_value_types_with_nulls(dtype):
    rng = np.random.default_rng(11)
    n = 120_000
    k = rng.integers(0, 700, n).astype(np.int32)
    v = _values(dtype, n, rng)
    valid = rng.random(n) >= 0.15
    T.assert_parity([HostCol(k)], [(HostCol(v, valid), sorted_aggs())])


@pytest.mark.parametrize("tid,dtype", [(TypeId.TIMESTAMP_SECONDS, np.int64), (TypeId.DURATION_DAYS, np.int32),
                                       (TypeId.DECIMAL64, np.int64), (TypeId.DECIMAL32, np.int32)])
def test_chrono_and_decimal_values(tid, dtype):
    """NUNIQUE and NTH_ELEMENT take any fixed-width value (the others need
    arithmetic types)."""
    rng = np.random.default_rng(12)
    n = 60_000
    k = rng.integers(0, 300, n).astype(np.int32)
    v = rng.integers(-500, 500, n).astype(dtype)
    valid = rng.random(n) >= 0.1
    scale = -2 if tid in (TypeId.DECIMAL32, TypeId.DECIMAL64) else 0
    T.assert_parity([HostCol(k)], [(HostCol(v, valid, type_id=tid, scale=scale), sorted_aggs(numeric=False))])


@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
@pytest.mark.parametrize("card", [50, 5_000, 200_000])
def test_every_strategy(strategy, card):
    rng = np.random.default_rng(13)
    n = 400_000
    k = rng.integers(0, card, n).astype(np.int64)
    v = rng.normal(0, 1, n)
    w = rng.integers(-30, 30, n).astype(np.int32)
    wvalid = rng.random(n) >= 0.2
    reqs = [(HostCol(v), sorted_aggs() + [(Kind.SUM, 0), (Kind.VARIANCE, 1)]),
            (HostCol(w, wvalid), [(Kind.MEDIAN, 0), (Kind.NUNIQUE, 0), (Kind.COUNT_VALID, 0)])]
    got, _ = T.assert_parity([HostCol(k)], reqs, strategy=strategy)
    # the partitioned path builds no global table to label rows with
    assert got["stats"]["strategy"] != Strategy.PARTITIONED


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_two_word_keys_with_null_keys(policy):
    rng = np.random.default_rng(14)
    n = 200_000
    a = rng.integers(0, 40, n).astype(np.int64)
    b = rng.integers(-20, 20, n).astype(np.int32)
    av = rng.random(n) >= 0.05
    bv = rng.random(n) >= 0.05
    v = rng.normal(10, 3, n).astype(np.float32)
    vv = rng.random(n) >= 0.1
    T.assert_parity([HostCol(a, av), HostCol(b, bv)], [(HostCol(v, vv), sorted_aggs())], policy)


def test_dictionary_values():
    rng = np.random.default_rng(15)
    n = 100_000
    k = rng.integers(0, 400, n).astype(np.int32)
    dk = np.unique(rng.normal(0, 100, 2000))
    idx = rng.integers(0, len(dk), n).astype(np.int32)
    valid = rng.random(n) >= 0.1
    vals = HostCol(idx, valid, dict_keys=HostCol(dk))
    T.assert_parity([HostCol(k)], [(vals, sorted_aggs())])


def test_many_rows_few_groups_and_many_groups():
    """Many radix tiles (4,096 records each) and label widths over 16 bits."""
    rng = np.random.default_rng(16)
    n = 2_000_000
    for card in (3, 300_000):
        k = rng.integers(0, card, n).astype(np.int32)
        v = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64)
        T.assert_parity([HostCol(k)], [(HostCol(v), [(Kind.MEDIAN, 0), (Kind.NUNIQUE, 0),
                                                     (Kind.QUANTILE, 0, {"quantiles": [0.01, 0.99],
                                                                         "interpolation": 3}),
                                                     (Kind.NTH_ELEMENT, -2, {"null_policy": 1})])],
                        threads=8)


def test_all_null_values_and_empty_input():
    k = np.array([1, 2, 1, 3], np.int32)
    v = np.array([1.0, 2.0, 3.0, 4.0])
    T.assert_parity([HostCol(k)], [(HostCol(v, np.zeros(4, bool)), sorted_aggs())])
    e = np.zeros(0, np.int32)
    T.assert_parity([HostCol(e)], [(HostCol(np.zeros(0)), sorted_aggs())])


def test_null_keys_are_excluded_from_sorted_kinds():
    rng = np.random.default_rng(17)
    n = 50_000
    k = rng.integers(0, 100, n).astype(np.int16)
    kv = rng.random(n) >= 0.3
    v = rng.integers(0, 10, n).astype(np.int64)
    T.assert_parity([HostCol(k, kv)], [(HostCol(v), sorted_aggs())], NullPolicy.EXCLUDE)


@pytest.mark.parametrize("case", ["int64_full_range", "float64_unit_interval", "float32_no_neg_zero",
                                  "float64_wide", "constant_values", "tiny_range_many_groups"])
def test_record_formats(case):
    """Values whose range fits one 64-bit record beside the group label take
    the packed records, the others (full-range int64, wide float64, float32
    with -0.0) the split ones: both must give the oracle's results."""
    rng = np.random.default_rng(18)
    n, card = 150_000, 2_000
    if case == "int64_full_range":
        v = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64)
    elif case == "float64_unit_interval":
        v = 1.0 + rng.random(n)
    elif case == "float32_no_neg_zero":
        v = rng.normal(0, 1, n).astype(np.float32)
        v[v == 0] = 1.0
    elif case == "float64_wide":
        v = rng.normal(0, 1e100, n)
    elif case == "constant_values":
        v = np.full(n, 7, np.int32)
    else:
        card = 60_000
        v = rng.integers(0, 3, n).astype(np.int16)
    k = rng.integers(0, card, n).astype(np.int32)
    valid = rng.random(n) >= 0.1
    aggs = sorted_aggs()
    if case == "int64_full_range":
        # the groups' int64 sums wrap: the reference's M2 is then taken about
        # the wrapped mean, this library's about the true one (a documented
        # edge shared with VARIANCE), so M2 is left out here
        aggs = [a for a in aggs if a[0] != Kind.M2]
    T.assert_parity([HostCol(k)], [(HostCol(v, valid), aggs)])
