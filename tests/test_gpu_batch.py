"""Parity of the batched groupby (gbx_batch_*): every instance of a batch must
give what the oracle gives on that instance alone, in every table mode, with
uneven row counts and cardinalities, nulls, several channels, empty
instances, a re-plan after a table overflow, input refills between executes
and rebinding; the tuner's table must persist and be read back."""
from __future__ import annotations

import os

import numpy as np
import pytest

from cudf_b200._abi import BatchMode, Kind, NullPolicy, Tune
from cudf_b200.workloads import batched_instance, batched_spec
from oracle.oracle import HostCol
from tests.gbx_testing import assert_parity, compare_keys, device_column, run_gpu, sort_order

pytestmark = pytest.mark.gpu

SUM_COUNT_MAX = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MAX, 0)]
MODES = [BatchMode.AUTO, BatchMode.SHARED, BatchMode.WARP, BatchMode.GLOBAL]


def device_instances(insts):
    from cudf_b200 import BatchInstance, GroupByRequest, Table
    from cudf_b200.aggregation import Aggregation

    out = []
    for keys, reqs in insts:
        kt = Table([device_column(k) for k in keys])
        rq = [GroupByRequest(device_column(v), [Aggregation(Kind(k), d) for k, d in aggs]) for v, aggs in reqs]
        out.append(BatchInstance(kt, rq))
    return out


def run_batch(insts, null_policy=NullPolicy.EXCLUDE, **kw):
    from cudf_b200 import BatchGroupBy

    kw.setdefault("tune", Tune.OFF)
    dev = device_instances(insts)
    b = BatchGroupBy(dev, null_handling=null_policy, **kw)
    return b, dev, b.execute()


def host_of(res):
    keys = [(int(c.type_id),) + tuple(c.to_numpy()) for c in res.keys.columns()]
    results = [[(int(c.type_id),) + tuple(c.to_numpy()) for c in t.columns()] for t in res.results]
    return keys, results


def instance_view(keys, results, offsets, i):
    b, e = int(offsets[i]), int(offsets[i + 1])

    def sl(t):
        return (t[0], t[1][b:e], None if t[2] is None else t[2][b:e])

    return {"num_groups": e - b, "keys": [sl(k) for k in keys], "results": [[sl(r) for r in q] for q in results]}


def check_batch(insts, res, null_policy=NullPolicy.EXCLUDE):
    keys, results = host_of(res)
    assert len(res.offsets) == len(insts) + 1 and res.offsets[0] == 0
    assert np.all(np.diff(res.offsets) >= 0)
    for i, (k, reqs) in enumerate(insts):
        assert_parity(k, reqs, null_policy, gpu=instance_view(keys, results, res.offsets, i))


def uneven(n_inst, rows_range=(100, 20_000), card_range=(10, 3_000), seed=11, aggs=SUM_COUNT_MAX):
    spec = batched_spec(n_inst, rows_range, card_range, seed=seed)
    insts = []
    for i in range(n_inst):
        k, v = batched_instance(spec, i)
        insts.append(([HostCol(k)], [(HostCol(v), aggs)]))
    return insts


@pytest.mark.parametrize("mode", MODES, ids=lambda m: m.name)
def test_uneven_instances_every_mode(mode):
    insts = uneven(40)
    b, _, res = run_batch(insts, force_mode=mode)
    check_batch(insts, res)
    st = b.stats()
    assert st["num_instances"] == 40 and st["num_groups"] == res.num_groups
    assert st["kernels_per_execute"] >= 4
    assert st["aggregate_ms"] > 0 and st["execute_ms"] >= st["aggregate_ms"]
    plan = b.instance_plan()
    if mode != BatchMode.AUTO:
        # a shared-memory mode falls back to the global table only when it does not fit
        assert np.all((plan["mode"] == int(mode)) | (plan["mode"] == int(BatchMode.GLOBAL)))
        assert (plan["mode"] == int(mode)).any()


@pytest.mark.parametrize("one_shot", [False, True], ids=["graph", "one_shot"])
@pytest.mark.parametrize("block", [256, 512])
@pytest.mark.parametrize("tile", [1024, 5000])
def test_block_shapes_small_tiles_and_one_shot(block, tile, one_shot):
    insts = uneven(24, rows_range=(1_000, 40_000), card_range=(5, 800), seed=12)
    b, _, res = run_batch(insts, block_threads=block, tile_rows=tile, one_shot=one_shot)
    check_batch(insts, res)
    assert b.stats()["block_threads"] == block
    check_batch(insts, b.execute())  # a second execute gives the same groups


def _mixed_instances(n_inst, seed, policy_nulls=True, empty_every=7):
    rng = np.random.default_rng(seed)
    insts = []
    for i in range(n_inst):
        n = 0 if i % empty_every == 3 else int(10 ** rng.uniform(1, 4.3))
        card = int(10 ** rng.uniform(0.5, 3.5))
        k1 = rng.integers(0, card, n, dtype=np.int32)
        k2 = rng.integers(-3, 3, n, dtype=np.int16)
        kv1 = (rng.random(n) > 0.05) if (policy_nulls and i % 2 == 0) else None
        kv2 = (rng.random(n) > 0.03) if (policy_nulls and i % 3 == 0) else None
        a = rng.integers(-1_000_000, 1_000_000, n, dtype=np.int64)
        f = rng.standard_normal(n).astype(np.float32)
        fv = (rng.random(n) > 0.1) if i % 4 != 1 else None
        insts.append((
            [HostCol(k1, kv1), HostCol(k2, kv2)],
            [(HostCol(a), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1), (Kind.COUNT_ALL, 0)]),
             (HostCol(f, fv), [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MAX, 0), (Kind.STD, 0), (Kind.MEAN, 0)])],
        ))
    return insts


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
@pytest.mark.parametrize("mode", MODES, ids=lambda m: m.name)
def test_composite_keys_nulls_and_empty_instances(policy, mode):
    insts = _mixed_instances(30, seed=21)
    _, _, res = run_batch(insts, null_policy=policy, force_mode=mode)
    check_batch(insts, res, policy)


def test_same_result_alone_and_in_the_batch():
    """Each instance's batch result equals the plain groupby on it alone."""
    insts = _mixed_instances(12, seed=22)
    _, _, res = run_batch(insts, null_policy=NullPolicy.INCLUDE)
    keys, results = host_of(res)
    for i, (k, reqs) in enumerate(insts):
        if len(k[0].values) == 0:
            continue
        alone = run_gpu(k, reqs, NullPolicy.INCLUDE)
        mixed = instance_view(keys, results, res.offsets, i)
        assert alone["num_groups"] == mixed["num_groups"]
        go, ao = sort_order(mixed["keys"]), sort_order(alone["keys"])
        compare_keys(mixed["keys"], alone["keys"], go, ao)
        for q in range(len(reqs)):
            for a in range(len(reqs[q][1])):
                _, gv, gm = mixed["results"][q][a]
                _, av, am = alone["results"][q][a]
                gmask = np.ones(len(gv), bool) if gm is None else gm
                amask = np.ones(len(av), bool) if am is None else am
                assert np.array_equal(gmask[go], amask[ao])
                x, y = np.asarray(gv)[go][amask[ao]], np.asarray(av)[ao][amask[ao]]
                if x.dtype.kind == "f":
                    # float32 inputs, float64 accumulation: |Δ| within 1e-12 of the group's sum |x| (≤ rows × 10)
                    assert np.all(np.abs(x.astype(np.float64) - y.astype(np.float64)) <= 1e-12 * 10 * len(k[0].values)
                                  + np.abs(y.astype(np.float64)) * 2.0 ** -23)
                else:
                    assert np.array_equal(x, y)


def test_overflow_replans_the_instance():
    """An instance whose sampled rows repeat one key while the rest are all
    distinct gets a table sized for the sample; the overflow re-plans it."""
    m = 2048
    n = 200_000
    keys = np.arange(1, n + 1, dtype=np.int64) * 7
    pos = ((np.arange(m) + 0.5) * n / m).astype(np.int64)
    keys[pos] = 0
    v = np.ones(n, dtype=np.int64)
    aggs = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0)]
    insts = [([HostCol(keys)], [(HostCol(v), aggs)])]
    insts += [([HostCol(k[0].values.astype(np.int64))], r) for k, r in uneven(5, seed=31, aggs=aggs)]
    b, _, res = run_batch(insts, force_mode=BatchMode.SHARED)
    check_batch(insts, res)
    assert b.stats()["retries"] >= 1
    # re-planned for its rows: the estimate is the row count, the table holds every row
    plan = b.instance_plan()
    assert plan["estimated_groups"][0] == n
    if plan["mode"][0] == int(BatchMode.GLOBAL):
        assert plan["table_slots"][0] >= n


def test_refill_inputs_between_executes_and_rebind():
    insts = uneven(10, seed=41)
    b, dev, res1 = run_batch(insts)
    check_batch(insts, res1)
    # refill every instance's key and value buffers in place (same sizes)
    rng = np.random.default_rng(5)
    new = []
    for (keys, reqs), d in zip(insts, dev):
        n = len(keys[0].values)
        k = rng.integers(0, 50, n, dtype=np.int32)
        v = rng.integers(0, 1000, n, dtype=np.int64)
        if n:
            d.keys[0].data.copy_(device_column(HostCol(k)).data)
            d.requests[0].values.data.copy_(device_column(HostCol(v)).data)
        new.append(([HostCol(k)], [(HostCol(v), reqs[0][1])]))
    check_batch(new, b.execute())
    # rebind to separate buffers of the same shapes
    rng = np.random.default_rng(6)
    other = []
    for keys, reqs in uneven(10, seed=41):
        k = rng.integers(0, 20, len(keys[0].values), dtype=np.int32)
        other.append(([HostCol(k)], reqs))
    b.rebind(device_instances(other))
    check_batch(other, b.execute())


def test_rebind_rejects_new_nulls():
    from cudf_b200 import LogicError

    insts = uneven(3, seed=42)
    b, _, _ = run_batch(insts)
    with_nulls = [([HostCol(k[0].values, np.arange(len(k[0].values)) % 5 != 0)], reqs) for k, reqs in insts]
    with pytest.raises(LogicError):
        b.rebind(device_instances(with_nulls))


def test_tuner_measures_persists_and_reuses(tmp_path):
    path = str(tmp_path / "tune.txt")
    insts = uneven(32, rows_range=(5_000, 60_000), card_range=(10, 3_000), seed=51)
    b1, _, res = run_batch(insts, tune=Tune.MISSING, tune_file=path)
    check_batch(insts, res)
    s1 = b1.stats()
    assert s1["classes_measured"] >= 1 and s1["classes_cached"] == 0
    lines = [l for l in open(path).read().splitlines() if l.strip()]
    assert len(lines) == 2 * s1["classes"]  # every class under both block shapes
    b2, _, res2 = run_batch(insts, tune=Tune.MISSING, tune_file=path)
    s2 = b2.stats()
    assert s2["classes_measured"] == 0 and s2["classes_cached"] == 2 * s2["classes"]
    check_batch(insts, res2)
    assert os.path.getsize(path) == sum(len(l) + 1 for l in lines)  # nothing appended


def test_dictionary_values_in_a_batch():
    rng = np.random.default_rng(61)
    insts = []
    for i in range(6):
        n = int(rng.integers(10, 5000))
        k = rng.integers(0, 40, n, dtype=np.int64)
        dk = HostCol(rng.standard_normal(17))
        idx = rng.integers(0, 17, n, dtype=np.int32)
        insts.append(([HostCol(k)], [(HostCol(idx, dict_keys=dk), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.MEAN, 0)])]))
    _, _, res = run_batch(insts)
    check_batch(insts, res)
