"""GPU parity: libgbx vs the oracle on the same seeded inputs, through the C ABI.

Sizes are chosen so the single-threaded oracle finishes in seconds; every
strategy (privatised shared-memory tables, global table) is exercised on every
workload shape.  Tolerances are those stated in tests/gbx_testing.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200 import workloads as W
from cudf_b200._abi import Kind, NullPolicy, Strategy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

ALL6 = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1)]
STRATS = [Strategy.AUTO, Strategy.PRIVATIZED, Strategy.GLOBAL, Strategy.WARP, Strategy.PARTITIONED,
          Strategy.BUCKETED]


def hc(a, v=None, **kw):
    return HostCol(a, v, **kw)


@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
def test_plain_10m_shape(strategy):
    d = W.plain_10m(n=300_000)
    aggs = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MEAN, 0), (Kind.MIN, 0), (Kind.MAX, 0)]
    T.assert_parity([hc(d.keys[0])], [(hc(d.values[0]), aggs)], strategy=strategy)


@pytest.mark.parametrize("card", [100, 10_000, 1_000_000])
@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
def test_plain_100m_shape(card, strategy):
    d = W.plain_100m(card, n=1_000_000)
    reqs = [(hc(d.values[0]), ALL6), (hc(d.values[1], d.value_valid[1]), ALL6)]
    got, want = T.assert_parity([hc(d.keys[0])], reqs, strategy=strategy)
    if strategy == Strategy.WARP and card == 100:
        assert got["stats"]["strategy"] == Strategy.WARP
    if strategy == Strategy.AUTO and card == 100:
        assert got["stats"]["strategy"] == Strategy.PRIVATIZED


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
def test_plain_200m_shape(policy, strategy):
    d = W.plain_200m(n=400_000, ranks=20_000)
    keys = [hc(d.keys[0], d.key_valid[0]), hc(d.keys[1], d.key_valid[1])]
    T.assert_parity(keys, [(hc(d.values[0]), [(Kind.SUM, 0), (Kind.MEAN, 0)])], policy, strategy)


@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
def test_empty_key_sentinel_collision(strategy):
    """int64 key -1 is the all-ones word the tables use as their empty marker."""
    rng = np.random.default_rng(7)
    k = rng.integers(-3, 3, size=50_000).astype(np.int64)
    k[::7] = -1
    v = rng.integers(-100, 100, size=50_000).astype(np.int64)
    T.assert_parity([hc(k)], [(hc(v), ALL6)], strategy=strategy)


@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
def test_two_word_keys(strategy):
    """(int64, int64) keys need two 64-bit table words (128-bit CAS path)."""
    rng = np.random.default_rng(8)
    n = 200_000
    a = rng.integers(0, 50, size=n).astype(np.int64)
    b = rng.integers(-5, 5, size=n).astype(np.int64)
    b[::11] = -1
    a[::13] = -1
    v = rng.standard_normal(n)
    T.assert_parity([hc(a), hc(b)], [(hc(v), ALL6)], strategy=strategy)


def test_two_word_keys_with_nulls_include():
    """(int64, int32) keys with a null bit each: 96 value bits + 2 null bits."""
    rng = np.random.default_rng(9)
    n = 100_000
    a = rng.integers(0, 30, size=n).astype(np.int64)
    b = rng.integers(0, 30, size=n).astype(np.int32)
    va = rng.random(n) > 0.1
    vb = rng.random(n) > 0.1
    v = rng.integers(0, 1000, size=n).astype(np.int32)
    T.assert_parity([hc(a, va), hc(b, vb)], [(hc(v), ALL6)], NullPolicy.INCLUDE)
    T.assert_parity([hc(a, va), hc(b, vb)], [(hc(v), ALL6)], NullPolicy.EXCLUDE)


def test_keys_wider_than_128_bits():
    """Two nullable int64 keys need 130 packed bits: the rows are labelled
    by a representative-row table and grouped on the label."""
    n = 1000
    a = np.arange(n, dtype=np.int64) % 37
    va = np.arange(n) % 3 > 0
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([hc(a, va), hc(a * 3, va)], [(hc(a), [(Kind.SUM, 0)])], policy)


def test_all_distinct_and_all_equal_keys():
    n = 300_000
    v = np.random.default_rng(10).standard_normal(n)
    T.assert_parity([hc(np.arange(n, dtype=np.int64))], [(hc(v), ALL6)])
    T.assert_parity([hc(np.full(n, 42, dtype=np.int32))], [(hc(v), ALL6)])


def test_all_keys_null():
    n = 10_000
    k = np.arange(n, dtype=np.int32)
    v = np.ones(n, dtype=np.float64)
    T.assert_parity([hc(k, np.zeros(n, bool))], [(hc(v), ALL6)])
    T.assert_parity([hc(k, np.zeros(n, bool))], [(hc(v), ALL6)], NullPolicy.INCLUDE)


def test_float_keys_nan_and_signed_zero():
    rng = np.random.default_rng(11)
    n = 100_000
    k = rng.integers(0, 20, size=n).astype(np.float64)
    k[::5] = np.nan
    k[1::9] = -0.0
    k[2::9] = 0.0
    k32 = k.astype(np.float32)
    v = rng.integers(0, 100, size=n).astype(np.int64)
    T.assert_parity([hc(k)], [(hc(v), ALL6)])
    T.assert_parity([hc(k32)], [(hc(v), ALL6)])


def test_float_values_with_nan_and_inf():
    rng = np.random.default_rng(12)
    n = 100_000
    k = rng.integers(0, 50, size=n).astype(np.int32)
    v = rng.standard_normal(n)
    v[::1000] = np.nan
    v[k == 3] = np.nan  # a group whose values are all NaN
    v[(k == 4) & (np.arange(n) % 2 == 0)] = np.inf
    T.assert_parity([hc(k)], [(hc(v), [(Kind.MIN, 0), (Kind.MAX, 0), (Kind.COUNT_VALID, 0)])])


def test_dictionary_keys_and_values():
    rng = np.random.default_rng(13)
    n = 100_000
    dict_vals = np.array([5, -3, 17, 1 << 40, 0, -9], dtype=np.int64)
    idx = rng.integers(0, len(dict_vals), size=n).astype(np.int32)
    vvalid = rng.random(n) > 0.05
    values = hc(idx, vvalid, dict_keys=hc(dict_vals))
    kidx = rng.integers(0, 40, size=n).astype(np.int32)
    keys = hc(kidx, dict_keys=hc(np.arange(40, dtype=np.int64) * 3))
    T.assert_parity([keys], [(values, ALL6 + [(Kind.SUM_OF_SQUARES, 0)])])


@pytest.mark.parametrize("tid", [TypeId.INT8, TypeId.INT16, TypeId.UINT8, TypeId.UINT16, TypeId.UINT32,
                                 TypeId.UINT64, TypeId.BOOL8, TypeId.FLOAT32])
def test_value_types(tid):
    rng = np.random.default_rng(14 + int(tid))
    n = 100_000
    k = rng.integers(0, 300, size=n).astype(np.int16)
    from cudf_b200.column import storage_dtype
    if tid == TypeId.FLOAT32:
        v = rng.standard_normal(n).astype(np.float32)
    elif tid == TypeId.BOOL8:
        v = (rng.random(n) > 0.5).astype(np.uint8)
    else:
        dt = storage_dtype(tid)
        info = np.iinfo(dt)
        v = rng.integers(info.min, info.max, size=n, endpoint=True, dtype=dt)
        if tid == TypeId.UINT64:
            # keep per-group sums below 2^63: libcudf derives MEAN/VAR of an
            # integer column from its INT64 SUM, which wraps beyond that
            v = v >> np.uint64(24)
    valid = rng.random(n) > 0.2
    aggs = ALL6 + [(Kind.SUM_OF_SQUARES, 0), (Kind.COUNT_ALL, 0), (Kind.STD, 0)]
    T.assert_parity([hc(k)], [(hc(v, valid, type_id=tid), aggs)])


def test_product_and_sum_of_squares():
    rng = np.random.default_rng(15)
    n = 50_000
    k = rng.integers(0, 1000, size=n).astype(np.int32)
    vi = rng.integers(-3, 4, size=n).astype(np.int64)
    vf = rng.uniform(0.9, 1.1, size=n)
    aggs = [(Kind.PRODUCT, 0), (Kind.SUM_OF_SQUARES, 0)]
    T.assert_parity([hc(k)], [(hc(vi), aggs), (hc(vf), aggs)])


def test_durations_and_decimals():
    rng = np.random.default_rng(16)
    n = 50_000
    k = rng.integers(0, 100, size=n).astype(np.int64)
    d = rng.integers(-10**6, 10**6, size=n).astype(np.int64)
    dec = rng.integers(-10**4, 10**4, size=n).astype(np.int32)
    aggs = [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0), (Kind.COUNT_VALID, 0)]
    T.assert_parity([hc(k)], [(hc(d, type_id=TypeId.DURATION_SECONDS), aggs),
                              (hc(dec, type_id=TypeId.DECIMAL32, scale=-2), aggs)])


def test_var_ddof_and_large_offset_values():
    """VAR with ddof 0/1/2 on values with a mean far from zero (the shifted sums
    keep precision where sum(x^2) - n mean^2 would cancel)."""
    rng = np.random.default_rng(17)
    n = 200_000
    k = rng.integers(0, 200, size=n).astype(np.int32)
    v = 1e9 + rng.standard_normal(n)
    aggs = [(Kind.VARIANCE, 0), (Kind.VARIANCE, 1), (Kind.VARIANCE, 2), (Kind.STD, 1)]
    for s in STRATS:
        T.assert_parity([hc(k)], [(hc(v), aggs)], strategy=s)


def test_sliced_columns():
    """Column views with a row offset (cudf::slice) on keys, values and masks."""
    from cudf_b200 import Column, GroupBy, GroupByRequest, Table, aggregation as agg
    from oracle import oracle as orc

    rng = np.random.default_rng(18)
    n = 10_000
    k = rng.integers(0, 50, size=n).astype(np.int32)
    kv = rng.random(n) > 0.1
    v = rng.standard_normal(n)
    vv = rng.random(n) > 0.1
    b, e = 37, 9_001
    kc = Column.from_numpy(k, kv).slice(b, e)
    vc = Column.from_numpy(v, vv).slice(b, e)
    gb = GroupBy(Table([kc]))
    kt, res = gb.aggregate([GroupByRequest(vc, [agg.sum(), agg.count(), agg.max()])])
    got = {"num_groups": kt.num_rows(), "keys": [(int(kt[0].type_id),) + kt[0].to_numpy()],
           "results": [[(int(c.type_id),) + c.to_numpy() for c in res[0].columns()]]}
    reqs = [(hc(v[b:e], vv[b:e]), [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MAX, 0)])]
    T.assert_parity([hc(k[b:e], kv[b:e])], reqs, gpu=got)


def test_overflowing_estimate_retries():
    """Keys chosen so the strided sample sees one key while the data has ~1M
    groups: the first table overflows and the call retries with a larger one."""
    n = 1_000_000
    k = np.arange(n, dtype=np.int64) + 10
    nsample = 1 << 16
    pos = ((np.arange(nsample) + 0.5) * n / nsample).astype(np.int64)
    k[pos] = 0
    v = np.ones(n, dtype=np.int64)
    got, _ = T.assert_parity([hc(k)], [(hc(v), [(Kind.SUM, 0), (Kind.COUNT_VALID, 0)])])
    assert got["stats"]["retries"] >= 1


def test_many_requests_and_duplicates():
    rng = np.random.default_rng(19)
    n = 100_000
    k = rng.integers(0, 500, size=n).astype(np.int32)
    v1 = rng.standard_normal(n)
    v2 = rng.integers(0, 10, size=n).astype(np.int32)
    reqs = [(hc(v1), [(Kind.SUM, 0), (Kind.SUM, 0), (Kind.MEAN, 0)]), (hc(v1), [(Kind.MAX, 0)]),
            (hc(v2), [(Kind.COUNT_ALL, 0), (Kind.VARIANCE, 0)]), (hc(v2), [])]
    T.assert_parity([hc(k)], reqs)


def test_empty_input_types():
    k = np.zeros(0, np.int64)
    v = np.zeros(0, np.float32)
    got = T.run_gpu([hc(k)], [(hc(v), ALL6)])
    assert got["num_groups"] == 0
    types = [r[0] for r in got["results"][0]]
    assert types == [TypeId.FLOAT32, TypeId.INT32, TypeId.FLOAT32, TypeId.FLOAT32, TypeId.FLOAT64, TypeId.FLOAT64]


@pytest.mark.parametrize("card", [1_000, 100_000, 3_000_000])
def test_partitioned_bucket_and_slice_modes(card):
    """Partitioned strategy: few large buckets (split across warps, merged in
    region tables) and many small buckets (written out directly)."""
    rng = np.random.default_rng(card)
    n = 2_000_000
    k = rng.integers(0, card, size=n).astype(np.int64)
    k[::101] = -1
    a = rng.integers(-1000, 1000, size=n).astype(np.int32)
    b = rng.standard_normal(n)
    bv = rng.random(n) > 0.2
    reqs = [(hc(a), ALL6), (hc(b, bv), ALL6)]
    got, _ = T.assert_parity([hc(k)], reqs, strategy=Strategy.PARTITIONED)
    assert got["stats"]["strategy"] == Strategy.PARTITIONED


@pytest.mark.parametrize("card", [3_000, 200_000])
def test_partitioned_every_kind_and_type(card):
    """Partitioned strategy on every aggregation kind and value type, eight
    channels (several register-fold passes per group), a dictionary value
    column and durations, with ~1.5 and ~100 rows per group."""
    rng = np.random.default_rng(24 + card)
    n = 300_000
    k = rng.integers(0, card, size=n).astype(np.int64)
    k[::97] = -1  # the all-ones key
    every = ALL6 + [(Kind.SUM_OF_SQUARES, 0), (Kind.COUNT_ALL, 0), (Kind.STD, 0), (Kind.VARIANCE, 0)]
    reqs = []
    for tid, dt in [(TypeId.INT8, np.int8), (TypeId.UINT16, np.uint16), (TypeId.UINT64, np.uint64)]:
        info = np.iinfo(dt)
        v = rng.integers(info.min, info.max, size=n, endpoint=True, dtype=dt)
        if tid == TypeId.UINT64:
            v = v >> np.uint64(24)  # per-group sums below 2^63, as in test_value_types
        reqs.append((hc(v, rng.random(n) > 0.2, type_id=tid), every))
    reqs.append((hc(rng.standard_normal(n).astype(np.float32), rng.random(n) > 0.1), every))
    reqs.append((hc(rng.integers(-3, 4, size=n).astype(np.int64)), [(Kind.PRODUCT, 0), (Kind.SUM, 0)]))
    reqs.append((hc(rng.uniform(0.9, 1.1, size=n)), [(Kind.PRODUCT, 0), (Kind.MIN, 0), (Kind.MAX, 0)]))
    dict_vals = np.array([5, -3, 17, 1 << 40, 0, -9], dtype=np.int64)
    idx = rng.integers(0, len(dict_vals), size=n).astype(np.int32)
    reqs.append((hc(idx, rng.random(n) > 0.05, dict_keys=hc(dict_vals)), ALL6))
    d = rng.integers(-10**6, 10**6, size=n).astype(np.int64)
    reqs.append((hc(d, type_id=TypeId.DURATION_SECONDS), [(Kind.SUM, 0), (Kind.MEAN, 0), (Kind.MAX, 0)]))
    got, _ = T.assert_parity([hc(k)], reqs, strategy=Strategy.PARTITIONED)
    assert got["stats"]["strategy"] == Strategy.PARTITIONED


@pytest.mark.parametrize("two_words", [False, True], ids=["one_word", "two_words"])
def test_partitioned_cta_tables(two_words):
    """~7.8M groups of ~1 row: one grouping table per CTA over 2^16 buckets
    (two radix passes, where warp tables would need 2^17 buckets and three),
    with the all-ones key, null keys kept (INCLUDE) and null values."""
    rng = np.random.default_rng(31 + two_words)
    n = 8_000_000
    a = rng.integers(0, 1 << 40, size=n).astype(np.int64)
    a[::89] = -1
    keys = [hc(a, rng.random(n) > 0.01)]
    if two_words:
        keys.append(hc(rng.integers(0, 3, size=n).astype(np.int32)))
    x = rng.integers(-1000, 1000, size=n).astype(np.int32)
    y = rng.standard_normal(n)
    reqs = [(hc(x), ALL6), (hc(y, rng.random(n) > 0.2), ALL6)]
    got, _ = T.assert_parity(keys, reqs, NullPolicy.INCLUDE, Strategy.PARTITIONED)
    st = got["stats"]
    assert (st["partition_bits"], st["retries"]) == (16, 0)
    assert st["bucket_slots"] >= 256


@pytest.mark.parametrize("card,bits", [(10_000, 8), (40_000, 16)])
def test_bucketed_chosen_for_mid_cardinality(card, bits):
    """5M rows over 1e4 / 4e4 groups: AUTO partitions the rows into buckets
    and groups tiles of the bucket-ordered rows in shared memory -- one radix
    pass (2^8 buckets) at 1e4; at 4e4 a CTA's run would meet ~290 groups, more
    than a 512-slot table holds at half load, so two passes (2^16)."""
    rng = np.random.default_rng(40 + card)
    n = 5_000_000
    k = rng.integers(0, card, size=n).astype(np.int64) * 7919 - 3
    a = rng.integers(-10**6, 10**6, size=n).astype(np.int64)
    b = rng.standard_normal(n).astype(np.float32)
    bv = rng.random(n) > 0.1
    got, _ = T.assert_parity([hc(k)], [(hc(a), ALL6), (hc(b, bv), ALL6)])
    st = got["stats"]
    assert (st["strategy"], st["partition_bits"], st["retries"]) == (Strategy.BUCKETED, bits, 0)


def test_partitioned_skewed_keys():
    """Zipf-skewed composite keys: one bucket holds a large share of the rows."""
    d = W.plain_200m(n=1_500_000, ranks=50_000)
    keys = [hc(d.keys[0], d.key_valid[0]), hc(d.keys[1], d.key_valid[1])]
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity(keys, [(hc(d.values[0]), [(Kind.SUM, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1)])], policy,
                        Strategy.PARTITIONED)


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_skewed_keys_stream_kernel(policy):
    """Zipf(1.5) keys over 50,000 ranks: AUTO keeps the hot keys in the
    streamed-tile kernel's shared tables and sends the rare keys' rows to the
    global table, so one group's partials arrive both ways (VAR shifts merged
    across them)."""
    rng = np.random.default_rng(31)
    n = 1_500_000
    ranks = 50_000
    w = np.arange(1, ranks + 1, dtype=np.float64) ** -1.5
    cdf = np.cumsum(w) / w.sum()
    j = np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), ranks - 1)
    key_of_rank = (rng.permutation(ranks) * 7 - 3).astype(np.int32)  # 33 packed bits with a null bit: one word
    k = key_of_rank[j]
    kvalid = rng.random(n) >= 0.01
    a = rng.integers(-1_000_000, 1_000_000, size=n).astype(np.int64)
    b = (1e6 + rng.standard_normal(n)).astype(np.float64)
    bvalid = rng.random(n) >= 0.2
    reqs = [(hc(a), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.COUNT_ALL, 0)]),
            (hc(b, bvalid), [(Kind.MEAN, 0), (Kind.VARIANCE, 1), (Kind.STD, 0), (Kind.COUNT_VALID, 0)])]
    got, _ = T.assert_parity([hc(k, kvalid)], reqs, policy)
    assert got["stats"]["strategy"] == Strategy.PRIVATIZED
