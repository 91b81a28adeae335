"""The served groupby (gbx_server_*): each result is the same alone and in
the mix -- against the oracle and against the plain form run alone -- with
requests merged into batched launches, admission held to the HBM budget,
oversized requests run alone, errors reported per request, and shutdown
with requests still waiting."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy
from oracle.oracle import HostCol
from tests.gbx_testing import FLOAT_RTOL, assert_parity, compare_keys, device_column, run_gpu, sort_order

pytestmark = pytest.mark.gpu

SUM_COUNT_MEAN = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MEAN, 0)]


def served_request(rng, rows, card):
    k = rng.integers(0, card, rows, dtype=np.int64)
    v = rng.standard_normal(rows)
    return [HostCol(k)], [(HostCol(v), SUM_COUNT_MEAN)]


def to_device(keys, reqs):
    from cudf_b200 import GroupByRequest, Table
    from cudf_b200.aggregation import Aggregation

    return (Table([device_column(k) for k in keys]),
            [GroupByRequest(device_column(v), [Aggregation(Kind(a), d) for a, d in aggs]) for v, aggs in reqs])


def host_result(kt, results):
    out = {"num_groups": kt.num_rows() if kt.num_columns() else 0, "keys": [], "results": []}
    for c in kt.columns():
        out["keys"].append((int(c.type_id),) + tuple(c.to_numpy()))
    for t in results:
        out["results"].append([(int(c.type_id),) + tuple(c.to_numpy()) for c in t.columns()])
    return out


def assert_same_as_alone(mixed, alone, rows_bound):
    """Groups, validity and integer results identical; floats within the
    summation bound FLOAT_RTOL * sum|x|, with sum|x| <= rows_bound * max|x|
    (the inputs here are N(0,1): max|x| < 10)."""
    assert mixed["num_groups"] == alone["num_groups"]
    go, ao = sort_order(mixed["keys"]), sort_order(alone["keys"])
    compare_keys(mixed["keys"], alone["keys"], go, ao)
    for q in range(len(alone["results"])):
        for a in range(len(alone["results"][q])):
            _, gv, gm = mixed["results"][q][a]
            _, av, am = alone["results"][q][a]
            gmask = np.ones(len(gv), bool) if gm is None else gm
            amask = np.ones(len(av), bool) if am is None else am
            assert np.array_equal(gmask[go], amask[ao])
            x, y = np.asarray(gv)[go][amask[ao]], np.asarray(av)[ao][amask[ao]]
            if x.dtype.kind != "f":
                assert np.array_equal(x, y)
            else:
                assert np.all(np.abs(x - y) <= FLOAT_RTOL * 10.0 * rows_bound)


def test_each_result_same_alone_and_in_the_mix():
    from cudf_b200 import Server

    rng = np.random.default_rng(7)
    sizes = [(int(10 ** rng.uniform(2, 5.3)), int(10 ** rng.uniform(1, 5))) for _ in range(40)]
    reqs = [served_request(rng, n, c) for n, c in sizes]
    srv = Server(workers=4, batch_max_rows=30_000, batch_max_requests=16)
    dev = [to_device(k, r) for k, r in reqs]
    tickets = [srv.submit(kt, rq) for kt, rq in dev]
    mixed = []
    for t in tickets:
        kt, res, timing = srv.wait(t)
        assert timing["done_s"] >= timing["admitted_s"] >= timing["submitted_s"]
        mixed.append(host_result(kt, res))
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    srv.close()
    for (k, r), m in zip(reqs, mixed):
        assert_parity(k, r, NullPolicy.EXCLUDE, gpu=m)
        assert_same_as_alone(m, run_gpu(k, r), len(k[0].values))


def test_small_requests_merge_behind_a_large_one():
    """One worker busy with a large request; the small ones that queue up
    behind it run as one batched launch, with the plain form's results."""
    from cudf_b200 import Server

    rng = np.random.default_rng(8)
    big = served_request(rng, 20_000_000, 1000)
    smalls = [served_request(rng, int(rng.integers(500, 20_000)), int(rng.integers(5, 3000))) for _ in range(12)]
    srv = Server(workers=1, batch_max_rows=50_000, batch_max_requests=64)
    dbig = to_device(*big)
    dsm = [to_device(k, r) for k, r in smalls]
    t_big = srv.submit(*dbig)
    ts = [srv.submit(kt, rq) for kt, rq in dsm]
    srv.wait(t_big)
    merged = 0
    for (k, r), t in zip(smalls, ts):
        kt, res, timing = srv.wait(t)
        merged = max(merged, timing["batched"])
        got = host_result(kt, res)
        assert_parity(k, r, NullPolicy.EXCLUDE, gpu=got)
        assert_same_as_alone(got, run_gpu(k, r), len(k[0].values))
    assert merged >= 2
    assert srv.stats()["batches"] >= 1
    srv.close()


def test_large_requests_run_one_at_a_time():
    """Requests of at least large_rows rows never overlap on the GPU (at most
    large_in_flight = 1 of them at once) while small ones still run beside
    them; every result matches the oracle."""
    from cudf_b200 import Server

    rng = np.random.default_rng(10)
    reqs = []
    for i in range(15):
        n = 300_000 if i % 3 == 0 else int(rng.integers(1000, 20_000))
        reqs.append(served_request(rng, n, int(rng.integers(10, 50_000))))
    srv = Server(workers=4, large_rows=200_000, large_in_flight=1)
    dev = [to_device(k, r) for k, r in reqs]
    ts = [srv.submit(kt, rq) for kt, rq in dev]
    spans = []
    for (k, r), t in zip(reqs, ts):
        kt, res, timing = srv.wait(t)
        if len(k[0].values) >= 200_000:
            spans.append((timing["admitted_s"], timing["done_s"]))
        assert_parity(k, r, NullPolicy.EXCLUDE, gpu=host_result(kt, res))
    srv.close()
    spans.sort()
    assert len(spans) == 5
    for (a0, d0), (a1, _) in zip(spans, spans[1:]):
        assert a1 >= d0, "two large requests were on the GPU at once"


def test_nullable_requests_merge_and_match():
    from cudf_b200 import Server

    rng = np.random.default_rng(9)
    reqs = []
    for i in range(16):
        n = int(rng.integers(1, 5000)) if i % 5 else 0
        k = rng.integers(0, 50, n, dtype=np.int32)
        kv = rng.random(n) > 0.1 if i % 2 else None
        v = rng.standard_normal(n).astype(np.float32)
        vv = rng.random(n) > 0.2 if i % 3 else None
        reqs.append(([HostCol(k, kv)], [(HostCol(v, vv), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.VARIANCE, 1),
                                                          (Kind.COUNT_ALL, 0)])]))
    srv = Server(workers=2, null_handling=NullPolicy.INCLUDE, batch_max_rows=10_000)
    dev = [to_device(k, r) for k, r in reqs]
    ts = [srv.submit(kt, rq) for kt, rq in dev]
    for (k, r), t in zip(reqs, ts):
        kt, res, _ = srv.wait(t)
        assert_parity(k, r, NullPolicy.INCLUDE, gpu=host_result(kt, res))
    srv.close()


def test_admission_holds_the_hbm_budget():
    from cudf_b200 import Server

    rng = np.random.default_rng(10)
    reqs = [served_request(rng, 200_000, 100) for _ in range(6)]
    dev = [to_device(k, r) for k, r in reqs]
    probe = Server(workers=1)
    t = probe.submit(*dev[0])
    _, _, timing = probe.wait(t)
    probe.close()
    charge = timing["reserved_bytes"]
    # room for one request at a time, though four workers are free
    srv = Server(workers=4, hbm_budget_bytes=int(charge * 1.5))
    ts = [srv.submit(kt, rq) for kt, rq in dev]
    for (k, r), t in zip(reqs, ts):
        kt, res, _ = srv.wait(t)
        assert_parity(k, r, NullPolicy.EXCLUDE, gpu=host_result(kt, res))
    st = srv.stats()
    assert st["max_in_flight"] == 1
    assert st["peak_reserved_bytes"] <= int(charge * 1.5)
    srv.close()
    # a request larger than the whole budget still runs (alone)
    srv = Server(workers=2, hbm_budget_bytes=int(charge // 4))
    t = srv.submit(*dev[1])
    kt, res, _ = srv.wait(t)
    assert_parity(*reqs[1], NullPolicy.EXCLUDE, gpu=host_result(kt, res))
    srv.close()


def test_errors_are_per_request():
    from cudf_b200 import Column, GroupByRequest, LogicError, Server, Table
    from cudf_b200.aggregation import Aggregation

    rng = np.random.default_rng(11)
    good = served_request(rng, 1000, 10)
    srv = Server(workers=2)
    # rejected at submit: values shorter than keys
    kt, rq = to_device(*good)
    short = Column.from_numpy(np.ones(10))
    with pytest.raises(LogicError):
        srv.submit(kt, [GroupByRequest(short, [Aggregation(Kind.SUM, 0)])])
    # fails while running: a dictionary index out of range
    idx = Column.from_numpy(np.array([0, 1, 7], dtype=np.int32))
    dk = Column.from_numpy(np.array([1.0, 2.0]))
    bad_keys = Table([Column.from_numpy(np.array([1, 1, 2], dtype=np.int64))])
    t_bad = srv.submit(bad_keys, [GroupByRequest(Column.dictionary(idx, dk), [Aggregation(Kind.SUM, 0)])])
    t_good = srv.submit(kt, rq)
    with pytest.raises(LogicError):
        srv.wait(t_bad)
    kt2, res, _ = srv.wait(t_good)
    assert_parity(*good, NullPolicy.EXCLUDE, gpu=host_result(kt2, res))
    assert srv.stats()["failed"] == 1
    srv.close()


def test_close_with_requests_waiting():
    from cudf_b200 import Server

    rng = np.random.default_rng(12)
    reqs = [served_request(rng, 2_000_000, 1000) for _ in range(6)]
    dev = [to_device(k, r) for k, r in reqs]
    srv = Server(workers=1)
    for kt, rq in dev:
        srv.submit(kt, rq)
    srv.close()  # the admitted request finishes, the waiting ones fail; no hang
