"""Shared helpers of the parity tests: build inputs once, run the oracle and
libgbx on them, sort both by key and compare.

Tolerances (stated here, used by every float comparison):
  * integer / byte / index results, keys, COUNT, validity: bit-exact;
  * float SUM/PRODUCT/SUM_OF_SQUARES/MEAN: |got - want| <= FLOAT_RTOL * scale + output
    rounding, where `scale` is sum(|x|) of the group's contributing values
    (the standard summation error bound), FLOAT_RTOL = 1e-12 for float64
    accumulation; float32 outputs add half an ulp of float32;
  * VAR/STD: |got - want| <= VAR_RTOL * (var + mean^2) (the bound of the
    shifted one-pass moments against a two-pass FP64 oracle), VAR_RTOL = 1e-9;
  * MIN/MAX: bit-exact (values are selected, not computed), NaN == NaN.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle.oracle import HostCol
from oracle import oracle as orc

FLOAT_RTOL = 1e-12
VAR_RTOL = 1e-9
KAT_RTOL = 1e-12  # known answers are exact rationals


def device_column(h: HostCol):
    """HostCol -> cudf_b200.Column on cuda:0 (same bytes)."""
    from cudf_b200 import Column

    if h.dict_keys is not None:
        idx = Column.from_numpy(h.values, h.valid)
        keys = device_column(h.dict_keys)
        return Column.dictionary(idx, keys)
    return Column.from_numpy(h.values, h.valid, type_id=h.type_id, scale=h.scale)


def run_gpu(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, strategy=None):
    """Runs libgbx; returns the same structure as oracle.groupby."""
    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200.aggregation import Aggregation

    kcols = [device_column(k) for k in keys]
    gb = GroupBy(Table(kcols), null_handling=null_policy)
    if strategy is not None:
        gb.set_strategy(strategy)
    reqs = [GroupByRequest(device_column(v), [Aggregation(Kind(k), d) for k, d in aggs]) for v, aggs in requests]
    ktab, results = gb.aggregate(reqs)
    out = {"num_groups": ktab.num_rows() if ktab.num_columns() else 0, "keys": [], "results": [], "stats": gb.last_stats()}
    for c in ktab.columns():
        v, m = c.to_numpy()
        out["keys"].append((int(c.type_id), v, m))
    for t in results:
        out["results"].append([(int(c.type_id),) + tuple(c.to_numpy()) for c in t.columns()])
    return out


def _sort_key_columns(keys):
    cols = []
    for tid, vals, valid in keys:
        v = np.asarray(vals)
        if v.dtype.kind == "f":
            v = np.where(np.isnan(v), np.inf, v)  # NaN keys sort last
            v = np.where(v == 0, 0.0, v)
        nul = np.zeros(len(v), dtype=np.int8) if valid is None else (~valid).astype(np.int8)
        vv = np.where(nul == 1, np.zeros(1, dtype=v.dtype), v)
        cols.append((nul, vv))
    return cols


def sort_order(keys) -> np.ndarray:
    cols = _sort_key_columns(keys)
    if not cols or len(cols[0][0]) == 0:
        return np.zeros(0, dtype=np.int64)
    seq = []
    for nul, vv in reversed(cols):
        seq.append(vv)
        seq.append(nul)
    return np.lexsort(seq)


def _valid_or_all(valid, n):
    return np.ones(n, dtype=bool) if valid is None else np.asarray(valid, dtype=bool)


def compare_keys(got_keys, want_keys, go, wo):
    assert len(got_keys) == len(want_keys)
    for (gt, gv, gm), (wt, wv, wm) in zip(got_keys, want_keys):
        assert gt == wt, f"key type {gt} != {wt}"
        n = len(wv)
        gmask = _valid_or_all(gm, n)[go]
        wmask = _valid_or_all(wm, n)[wo]
        assert np.array_equal(gmask, wmask), "key validity differs"
        a = np.asarray(gv)[go][wmask]
        b = np.asarray(wv)[wo][wmask]
        if a.dtype.kind == "f":
            a = np.where(a == 0, 0.0, a)
            b = np.where(b == 0, 0.0, b)
            assert np.array_equal(a, b, equal_nan=True), "keys differ"
        else:
            assert np.array_equal(a, b), "keys differ"


def compare_values(kind, got, want, go, wo, scale=None, var_scale=None, ctx=""):
    gt, gv, gm = got
    wt, wv, wm = want
    assert gt == wt, f"{ctx}: result type {TypeId(gt).name} != {TypeId(wt).name}"
    n = len(wv)
    assert len(gv) == n, f"{ctx}: length {len(gv)} != {n}"
    gmask = _valid_or_all(gm, n)[go]
    wmask = _valid_or_all(wm, n)[wo]
    assert np.array_equal(gmask, wmask), f"{ctx}: validity differs ({int((gmask != wmask).sum())} rows)"
    a = np.asarray(gv)[go][wmask]
    b = np.asarray(wv)[wo][wmask]
    if a.dtype.kind != "f":
        bad = np.nonzero(a != b)[0]
        assert len(bad) == 0, f"{ctx}: {len(bad)} integer results differ, first {a[bad[:3]]} vs {b[bad[:3]]}"
        return
    a64 = a.astype(np.float64)
    b64 = b.astype(np.float64)
    nan_ok = np.isnan(a64) == np.isnan(b64)
    assert nan_ok.all(), f"{ctx}: NaN placement differs"
    fin = ~np.isnan(b64)
    if kind in (Kind.MIN, Kind.MAX):
        assert np.array_equal(a64[fin], b64[fin]), f"{ctx}: min/max differ"
        return
    if kind in (Kind.VARIANCE, Kind.STD) and var_scale is not None:
        tol = VAR_RTOL * np.asarray(var_scale)[wo][wmask][fin] + 1e-300
        if kind == Kind.STD:
            # d(sqrt v) = dv / (2 sqrt v)
            tol = tol / np.maximum(2.0 * b64[fin], 1e-300)
            tol = np.maximum(tol, np.sqrt(VAR_RTOL * np.asarray(var_scale)[wo][wmask][fin]))
    elif scale is not None:
        tol = FLOAT_RTOL * np.asarray(scale)[wo][wmask][fin]
    elif kind == Kind.PRODUCT:
        tol = 1e-10 * np.abs(b64[fin])
    else:
        tol = KAT_RTOL * np.abs(b64[fin])
    if gt == TypeId.FLOAT32:
        tol = tol + np.abs(b64[fin]) * 2.0 ** -24 * 1.01
    diff = np.abs(a64[fin] - b64[fin])
    inf_same = np.isinf(b64[fin]) & (a64[fin] == b64[fin])
    bad = ~((diff <= tol) | inf_same)
    assert not bad.any(), (
        f"{ctx}: {int(bad.sum())} float results out of bound; worst rel "
        f"{float((diff[bad] / np.maximum(np.abs(b64[fin][bad]), 1e-300)).max()):.3e}")


def group_scales(keys: Sequence[HostCol], values: HostCol, null_policy) -> dict:
    """Per-group error scales in oracle group order, computed with the oracle
    itself: sum|x|, sum x^2, count and mean x^2 (= var_pop + mean^2)."""
    vals = values.values if values.dict_keys is None else values.dict_keys.values[values.values]
    x = vals.astype(np.float64)
    absx = HostCol(np.abs(x), values.valid)
    sq = HostCol(x * x, values.valid)
    r = orc.groupby(keys, [(absx, [(Kind.SUM, 0), (Kind.COUNT_VALID, 0)]), (sq, [(Kind.SUM, 0), (Kind.MEAN, 0)])],
                    null_policy)
    # the oracle is deterministic: same first-occurrence group order as the checked call
    f = lambda a: np.nan_to_num(np.asarray(a, dtype=np.float64), nan=0.0, posinf=0.0)
    return {"abs": f(r["results"][0][0][1]), "cnt": np.asarray(r["results"][0][1][1], dtype=np.float64),
            "sq": f(r["results"][1][0][1]), "msq": f(r["results"][1][1][1])}


def assert_parity(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, strategy=None, gpu=None):
    """Full parity check of libgbx against the oracle on the same inputs."""
    want = orc.groupby(keys, requests, null_policy)
    got = gpu if gpu is not None else run_gpu(keys, requests, null_policy, strategy)
    assert got["num_groups"] == want["num_groups"], f"groups {got['num_groups']} != {want['num_groups']}"
    go = sort_order(got["keys"])
    wo = sort_order(want["keys"])
    compare_keys(got["keys"], want["keys"], go, wo)
    for q, (vals, aggs) in enumerate(requests):
        vt = vals.dict_keys.type_id if vals.dict_keys is not None else vals.type_id
        is_float = vt in (TypeId.FLOAT32, TypeId.FLOAT64)
        sc = None
        for k, (kind, ddof) in enumerate(aggs):
            kind = Kind(kind)
            ctx = f"request {q} agg {kind.name}"
            s = v = None
            if kind in (Kind.VARIANCE, Kind.STD) or (is_float and kind in (Kind.SUM, Kind.MEAN, Kind.SUM_OF_SQUARES)):
                if sc is None:
                    sc = group_scales(keys, vals, null_policy)
                if kind == Kind.SUM:
                    s = sc["abs"]
                elif kind == Kind.MEAN:
                    s = sc["abs"] / np.maximum(sc["cnt"], 1)
                elif kind == Kind.SUM_OF_SQUARES:
                    s = sc["sq"]
                else:
                    v = sc["msq"]
            compare_values(kind, got["results"][q][k], want["results"][q][k], go, wo, s, v, ctx)
    return got, want
