"""GPU parity of ARGMIN / ARGMAX (libcudf's hash kinds, hash/groupby.cu:73-84;
update rule detail/aggregation/aggregation.cuh:436-491) against the oracle.

Every result is a row index (INT32), so parity is exact.  The reference's CAS
loop leaves ties and NaN order-dependent; this library and the oracle both
fix one order: the lowest row wins a tie, -0.0 ties +0.0, and NaN loses to
every number (an all-NaN group answers its first NaN row).  Values here are
drawn from small ranges so that ties are common.  Values of up to 32 bits
take every strategy (the ARG kinds become MIN / MAX of packed (order key, row)
words, gbx_args.cu); with a 64-bit value among them only the row-preserving
strategies (privatised shared table, global table) compute them, and a call
that forces another strategy runs on one of those two.
"""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, Strategy, TypeId
from cudf_b200.column import storage_dtype
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

ARGS = [(Kind.ARGMIN, 0), (Kind.ARGMAX, 0)]
STRATS = [Strategy.AUTO, Strategy.PRIVATIZED, Strategy.GLOBAL, Strategy.WARP, Strategy.PARTITIONED,
          Strategy.BUCKETED]
ROW_PRESERVING = {int(Strategy.PRIVATIZED), int(Strategy.GLOBAL)}


def _values(rng, tid, n):
    if tid in (TypeId.FLOAT32, TypeId.FLOAT64):
        return rng.integers(-20, 20, size=n).astype(storage_dtype(tid)) * 0.25
    dt = storage_dtype(tid)
    info = np.iinfo(dt)
    lo, hi = max(int(info.min), -40), min(int(info.max), 40)
    v = rng.integers(lo, hi, size=n, endpoint=True).astype(dt)
    if tid in (TypeId.INT64, TypeId.UINT64):
        # extremes of the type: the order key must keep their sign order
        v[::997] = info.max
        v[1::991] = info.min
    return v


@pytest.mark.parametrize("strategy", STRATS, ids=lambda s: s.name)
@pytest.mark.parametrize("tid", [TypeId.INT8, TypeId.INT16, TypeId.INT32, TypeId.INT64, TypeId.UINT32,
                                 TypeId.UINT64, TypeId.FLOAT32, TypeId.FLOAT64], ids=lambda t: t.name)
def test_value_types_and_strategies(tid, strategy):
    rng = np.random.default_rng(700 + int(tid))
    n = 60_000
    k = rng.integers(0, 500, size=n).astype(np.int32)
    v = _values(rng, tid, n)
    valid = rng.random(n) > 0.15
    got, _ = T.assert_parity([HostCol(k)], [(HostCol(v, valid, type_id=tid), ARGS + [(Kind.MIN, 0)]),
                                            (HostCol(v, type_id=tid), ARGS)], strategy=strategy)
    if storage_dtype(tid).itemsize == 8:
        assert got["stats"]["strategy"] in ROW_PRESERVING
    elif strategy in (Strategy.PARTITIONED, Strategy.BUCKETED, Strategy.GLOBAL, Strategy.PRIVATIZED):
        assert got["stats"]["strategy"] == int(strategy)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_float_specials(dt):
    """NaN, +-inf and both zeros; a group of only NaNs; a group of only zeros."""
    rng = np.random.default_rng(710)
    n = 50_000
    k = rng.integers(0, 40, size=n).astype(np.int64)
    v = rng.integers(-3, 4, size=n).astype(dt)
    v[::7] = np.nan
    v[3::11] = np.inf
    v[5::13] = -np.inf
    v[k == 5] = np.nan
    zeros = k == 6
    v[zeros] = np.where(np.arange(n)[zeros] % 2 == 0, dt(-0.0), dt(0.0))
    valid = rng.random(n) > 0.1
    T.assert_parity([HostCol(k)], [(HostCol(v, valid), ARGS + [(Kind.MIN, 0), (Kind.MAX, 0)])])


@pytest.mark.parametrize("strategy", [Strategy.AUTO, Strategy.PARTITIONED], ids=lambda s: s.name)
def test_high_cardinality_with_every_other_kind(strategy):
    """Beyond the shared tables: the global table, beside SUM/MEAN/VAR/... of
    the same channels (one 64-bit channel by CAS, one 32-bit one packed)."""
    rng = np.random.default_rng(711)
    n = 1_000_000
    k = rng.integers(0, 300_000, size=n, dtype=np.int64)
    a = rng.integers(-1000, 1000, size=n, endpoint=True).astype(np.int64)
    b = rng.integers(-50, 50, size=n).astype(np.float32)
    bv = rng.random(n) >= 0.10
    aggs = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0),
            (Kind.VARIANCE, 1)] + ARGS
    got, _ = T.assert_parity([HostCol(k)], [(HostCol(a), aggs), (HostCol(b, bv), aggs)], strategy=strategy)
    assert got["stats"]["strategy"] == int(Strategy.GLOBAL)


@pytest.mark.parametrize("strategy", [Strategy.AUTO, Strategy.PARTITIONED, Strategy.BUCKETED], ids=lambda s: s.name)
def test_high_cardinality_packed_args_partition(strategy):
    """Only 32-bit-or-narrower values: ARGMIN / ARGMAX ride the radix
    partitions as MIN / MAX of packed words (AUTO partitions at 3e5 groups)."""
    rng = np.random.default_rng(712)
    n = 2_000_000
    k = rng.integers(0, 600_000, size=n, dtype=np.int64)
    b = rng.integers(-50, 50, size=n).astype(np.float32)
    b[::101] = np.nan
    bv = rng.random(n) >= 0.10
    c = rng.integers(0, 7, size=n).astype(np.int16)
    aggs = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0)] + ARGS
    got, _ = T.assert_parity([HostCol(k)], [(HostCol(b, bv), aggs), (HostCol(c), ARGS + [(Kind.MAX, 0)])],
                             strategy=strategy)
    assert got["stats"]["strategy"] == int(Strategy.PARTITIONED if strategy == Strategy.AUTO else strategy)


def test_few_groups_many_ties():
    """1M rows into 3 groups of 2-valued data: every row ties the current
    holder, so the compare-and-swap loop and the packed minimum both run
    under full contention."""
    rng = np.random.default_rng(712)
    n = 1_000_000
    k = rng.integers(0, 3, size=n).astype(np.int32)
    a = rng.integers(0, 2, size=n).astype(np.int64)
    b = rng.integers(0, 2, size=n).astype(np.int16)
    T.assert_parity([HostCol(k)], [(HostCol(a), ARGS), (HostCol(b), ARGS)])


def test_dictionary_values_and_null_keys():
    rng = np.random.default_rng(713)
    n = 80_000
    dict_vals = np.array([5, -3, 17, 1 << 40, 0, -9, 5], dtype=np.int64)
    idx = rng.integers(0, len(dict_vals), size=n).astype(np.int32)
    vvalid = rng.random(n) > 0.05
    values = HostCol(idx, vvalid, dict_keys=HostCol(dict_vals))
    k = rng.integers(0, 200, size=n).astype(np.int32)
    kv = rng.random(n) > 0.05
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([HostCol(k, kv)], [(values, ARGS)], policy)


def test_sliced_columns_index_the_slice():
    """Row indices count from the sliced view's first row, as in the reference
    (the index is the source column_view's element index)."""
    from cudf_b200 import Column, GroupBy, GroupByRequest, Table, aggregation as agg

    rng = np.random.default_rng(714)
    n = 20_000
    k = rng.integers(0, 50, size=n).astype(np.int32)
    v = rng.integers(-100, 100, size=n).astype(np.int64)
    w = rng.integers(-100, 100, size=n).astype(np.int32)
    vv = rng.random(n) > 0.1
    b, e = 41, 15_003
    kc = Column.from_numpy(k).slice(b, e)
    gb = GroupBy(Table([kc]))
    kt, res = gb.aggregate([GroupByRequest(Column.from_numpy(v, vv).slice(b, e), [agg.argmin(), agg.argmax()]),
                            GroupByRequest(Column.from_numpy(w).slice(b, e), [agg.argmin(), agg.argmax()])])
    got = {"num_groups": kt.num_rows(), "keys": [(int(kt[0].type_id),) + kt[0].to_numpy()],
           "results": [[(int(c.type_id),) + c.to_numpy() for c in r.columns()] for r in res]}
    reqs = [(HostCol(v[b:e], vv[b:e]), ARGS), (HostCol(w[b:e]), ARGS)]
    T.assert_parity([HostCol(k[b:e])], reqs, gpu=got)


def test_served_requests_run_on_the_plain_path():
    """The served form keeps ARGMIN/ARGMAX requests out of its batched
    launches; each answer equals the oracle's."""
    from cudf_b200 import Server
    from tests.test_gpu_server import host_result, to_device

    rng = np.random.default_rng(715)
    reqs = []
    for i in range(8):
        n = int(rng.integers(100, 4000))
        k = rng.integers(0, 30, n, dtype=np.int64)
        v = rng.integers(-5, 5, n).astype(np.float64)
        reqs.append(([HostCol(k)], [(HostCol(v), ARGS + [(Kind.SUM, 0)])]))
    srv = Server(workers=2, batch_max_rows=10_000)
    dev = [to_device(k, r) for k, r in reqs]
    ts = [srv.submit(kt, rq) for kt, rq in dev]
    for (k, r), t in zip(reqs, ts):
        kt, res, _ = srv.wait(t)
        T.assert_parity(k, r, gpu=host_result(kt, res))
    srv.close()
