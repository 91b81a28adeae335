"""Full-size GPU parity: the benchmark's own groupby calls, at their real
sizes, checked against the oracle.

* 100M rows, int64 key of cardinality 1e6 and 1e8 (63.2M groups), int64 and
  float32-with-10%-nulls values, SUM/COUNT/MIN/MAX/MEAN/VAR on both -- the
  benchmark's cardinality-1e6 and 1e8 calls, through the public API.
* 200M rows, (int32, int16) key with 2% nulls per column, Zipf(1.2) over 1e5
  pairs (the hottest pair holds about a fifth of the rows), float64
  LogNormal(0, 1) value, SUM and MEAN, under both null policies.

Inputs come from the benchmark's device generators (cudf_b200.workloads);
they are copied to the host for the oracle, which runs with every host
thread.  Keys, COUNT and integer SUM/MIN/MAX are compared bit-exact after a
sort by key; floats within the bounds stated in tests/gbx_testing.py.  The
tolerance scales of the 100M-row calls come from numpy over the sorted rows
(the oracle's accumulators for 63.2M groups would not fit twice in host
memory).  Each case needs tens of GB of host memory and skips with that
reason when the host has less.
"""
from __future__ import annotations

import gc
import os

import numpy as np
import psutil
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle import oracle as orc
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

ALL6 = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1)]
THREADS = os.cpu_count() or 1


def _need_host_gb(gb):
    avail = psutil.virtual_memory().available / 2**30
    if avail < gb:
        pytest.skip(f"needs {gb} GB of free host memory, {avail:.0f} GB available")


def _gpu_result(kt, res):
    out = {"num_groups": kt.num_rows(), "keys": [], "results": []}
    for c in kt.columns():
        v, m = c.to_numpy()
        out["keys"].append((int(c.type_id), v, m))
    for t in res:
        out["results"].append([(int(c.type_id),) + tuple(c.to_numpy()) for c in t.columns()])
    return out


def _aggs():
    from cudf_b200.aggregation import Aggregation

    return [Aggregation(Kind(k), d) for k, d in ALL6]


@pytest.mark.parametrize("card", [1_000_000, 100_000_000], ids=["card1e6", "card1e8"])
def test_100m_rows_bench_call(card):
    _need_host_gb(48)
    import torch

    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200 import workloads as W

    n = 100_000_000
    dev = torch.device("cuda", 0)
    k, a, b = W.plain_100m_device(card, n, W.SEED0 + 2, dev)
    gb = GroupBy(Table([k]))
    kt, res = gb.aggregate([GroupByRequest(a, _aggs()), GroupByRequest(b, _aggs())])
    stats = gb.last_stats()
    got = _gpu_result(kt, res)
    kh = k.to_numpy()[0]
    cols = [a.to_numpy(), b.to_numpy()]
    del k, a, b, kt, res, gb
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    print(f"card {card:g}: {got['num_groups']} groups, strategy {stats['strategy']}, "
          f"partition bits {stats['partition_bits']}, bucket slots {stats['bucket_slots']}")

    go = T.sort_order(got["keys"])
    for q, (vals, valid) in enumerate(cols):
        want = orc.groupby([HostCol(kh)], [(HostCol(vals, valid), ALL6)], NullPolicy.EXCLUDE, THREADS)
        assert got["num_groups"] == want["num_groups"], f"groups {got['num_groups']} != {want['num_groups']}"
        wo = T.sort_order(want["keys"])
        T.compare_keys(got["keys"], want["keys"], go, wo)
        sc = T.sorted_group_scales(kh, vals, valid)
        # scales are in ascending key order; compare_values reads them in the
        # oracle's group order (position wo[i] holds sorted group i)
        inv = {}
        for name in ("abs", "cnt", "var"):
            arr = np.empty(len(wo))
            arr[wo] = sc[name]
            inv[name] = arr
        del sc
        is_float = vals.dtype.kind == "f"
        for j, (kind, ddof) in enumerate(ALL6):
            s = v = None
            if kind == Kind.VARIANCE:
                v = inv["var"]
            elif is_float and kind == Kind.SUM:
                s = inv["abs"]
            elif is_float and kind == Kind.MEAN:
                s = inv["abs"] / np.maximum(inv["cnt"], 1)
            T.compare_values(kind, got["results"][q][j], want["results"][0][j], go, wo, s, v,
                             ctx=f"card {card:g} request {q} {kind.name}")
        del want, wo, inv
        gc.collect()


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_200m_rows_zipf_composite_key(policy):
    _need_host_gb(32)
    import torch

    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200 import workloads as W

    n = 200_000_000
    dev = torch.device("cuda", 0)
    k1, k2, v = W.plain_200m_device(n, W.SEED0 + 3, dev)
    from cudf_b200.aggregation import Aggregation

    aggs = [(Kind.SUM, 0), (Kind.MEAN, 0)]
    gb = GroupBy(Table([k1, k2]), null_handling=policy)
    kt, res = gb.aggregate([GroupByRequest(v, [Aggregation(Kind(a), d) for a, d in aggs])])
    stats = gb.last_stats()
    got = _gpu_result(kt, res)
    host_keys = [HostCol(*k1.to_numpy()), HostCol(*k2.to_numpy())]
    vh = v.to_numpy()[0]
    del k1, k2, v, kt, res, gb
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    print(f"200M rows {policy.name}: {got['num_groups']} groups, strategy {stats['strategy']}")
    T.assert_parity(host_keys, [(HostCol(vh), aggs)], policy, gpu=got, threads=THREADS)
