"""Shared helpers of the parity tests: build inputs once, run the oracle and
libgbx on them, sort both by key and compare.

Tolerances (stated here, used by every float comparison):
  * integer / byte / index results, keys, COUNT, validity: bit-exact;
  * float SUM/PRODUCT/SUM_OF_SQUARES/MEAN: |got - want| <= FLOAT_RTOL * scale + output
    rounding, where `scale` is sum(|x|) of the group's contributing values
    (the standard summation error bound), FLOAT_RTOL = 1e-12 for float64
    accumulation; float32 outputs add half an ulp of float32;
  * VAR/STD: |got - want| <= VAR_EPS * n * (var + range^2), n the group's
    valid values, var its population variance, range = max - min, VAR_EPS =
    16 * 2^-52.  This is the rounding bound of the shifted one-pass moments
    (sum (x-K)^2 and sum (x-K) with K one of the group's values, so
    (mean - K)^2 <= range^2, each sum accurate to (n-1) 2^-53 of its
    magnitude) against a two-pass long-double oracle.  It scales with the
    variance, not with mean^2: sum x^2 - n mean^2 misses it by many orders of
    magnitude once |mean| >> std.  Integer columns beyond 2^53 add the
    rounding of their conversion to double, 4 * 2^-52 * max|x| * range.
    STD's bound is VAR's divided by 2 std (or its square root near 0);
  * MIN/MAX: bit-exact (values are selected, not computed), NaN == NaN.
  * M2: VAR's bound times the group's valid count (M2 = n VAR_pop);
  * MEDIAN/QUANTILE: equal to the oracle (the same double operations in the
    same order), NaN == NaN, +0.0 == -0.0; NUNIQUE / NTH_ELEMENT bit-exact.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle.oracle import HostCol
from oracle import oracle as orc
from oracle import presorted as orc_sorted
from oracle import structs as orc_structs

FLOAT_RTOL = 1e-12
VAR_EPS = 16.0 * 2.0 ** -52
KAT_RTOL = 1e-12  # known answers are exact rationals


def device_column(h: HostCol):
    """HostCol -> cudf_b200.Column on cuda:0 (same bytes, same offset and size)."""
    from cudf_b200 import Column

    if h.type_id == TypeId.STRUCT:
        n = h.children[0].size if h.children else 0
        valid = None if h.valid is None else np.asarray(h.valid, dtype=bool)[:n]
        col = Column.struct([device_column(m) for m in h.children], valid)
        if h.offset != 0 or h.size != n:
            col = col.slice(h.offset, h.offset + h.size)
        return col
    if h.type_id == TypeId.STRING:
        col = Column.from_strings(h.values, h.valid)
    elif h.dict_keys is not None:
        idx = Column.from_numpy(h.values, h.valid)
        keys = device_column(h.dict_keys)
        col = Column.dictionary(idx, keys)
    else:
        col = Column.from_numpy(h.values, h.valid, type_id=h.type_id, scale=h.scale)
    if h.offset != 0 or h.size != len(h.values):
        col = col.slice(h.offset, h.offset + h.size)
    return col


def _aggregation(a):
    """(kind, ddof[, extra]) -> cudf_b200.aggregation.Aggregation; extra holds
    null_policy / interpolation / quantiles."""
    from cudf_b200.aggregation import Aggregation

    extra = a[2] if len(a) > 2 else {}
    return Aggregation(Kind(a[0]), int(a[1]), null_policy=NullPolicy(extra.get("null_policy", 0)),
                       interpolation=extra.get("interpolation", 0), quantiles=tuple(extra.get("quantiles", ())))


def run_gpu(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, strategy=None,
            keys_are_sorted=False):
    """Runs libgbx; returns the same structure as oracle.groupby."""
    from cudf_b200 import GroupBy, GroupByRequest, Table
    from cudf_b200._abi import Sorted

    kcols = [device_column(k) for k in keys]
    gb = GroupBy(Table(kcols), null_handling=null_policy,
                 keys_are_sorted=Sorted.YES if keys_are_sorted else Sorted.NO)
    if strategy is not None:
        gb.set_strategy(strategy)
    reqs = [GroupByRequest(device_column(v), [_aggregation(a) for a in aggs]) for v, aggs in requests]
    ktab, results = gb.aggregate(reqs)
    out = {"num_groups": ktab.num_rows() if ktab.num_columns() else 0, "keys": [], "results": [], "stats": gb.last_stats()}
    for c in ktab.columns():
        out["keys"].append(_host_of(c))
    for t in results:
        out["results"].append([(int(c.type_id),) + tuple(c.to_numpy()) for c in t.columns()])
    return out


def _host_of(c):
    """(type_id, values, valid) of a result column; a STRUCT column's values
    are its members' (type_id, values, valid) over its rows."""
    if c.type_id == TypeId.STRUCT:
        _, valid = c.to_numpy()
        return (int(c.type_id), [_host_of(m.slice(c.offset, c.offset + c.size)) for m in c.children], valid)
    v, m = c.to_numpy()
    return (int(c.type_id), v, m)


def _sort_key_columns(keys):
    cols = []
    for tid, vals, valid in keys:
        v = np.asarray(vals)
        if v.dtype.kind == "f":
            v = np.where(np.isnan(v), np.inf, v)  # NaN keys sort last
            v = np.where(v == 0, 0.0, v)
        nul = np.zeros(len(v), dtype=np.int8) if valid is None else (~valid).astype(np.int8)
        if v.dtype == object:  # strings: nulls as ""
            vv = np.array(["" if n else x for x, n in zip(v, nul)], dtype=object)
            cols.append((nul, vv))
            continue
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


def rows_of_groups(order: np.ndarray, per_group: int) -> np.ndarray:
    """Result rows in the group order `order` when each group has
    `per_group` consecutive result rows (QUANTILE)."""
    order = np.asarray(order, dtype=np.int64)
    if per_group == 1:
        return order
    return (order[:, None] * per_group + np.arange(per_group)[None, :]).reshape(-1)


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


def compare_values(kind, got, want, go, wo, scale=None, var_scale=None, ctx="", exact=False):
    """Compares result columns row by row in the orders go / wo.  `exact`
    asks for equal floating values (NaN where NaN; +0.0 == -0.0)."""
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
    if exact:
        bad = np.nonzero(a64[fin] != b64[fin])[0]
        assert len(bad) == 0, f"{ctx}: {len(bad)} results differ, first {a64[fin][bad[:3]]} vs {b64[fin][bad[:3]]}"
        return
    if kind in (Kind.MIN, Kind.MAX):
        assert np.array_equal(a64[fin], b64[fin]), f"{ctx}: min/max differ"
        return
    if kind in (Kind.VARIANCE, Kind.STD, Kind.M2) and var_scale is not None:
        vtol = np.asarray(var_scale)[wo][wmask][fin] + 1e-300
        tol = vtol
        if kind == Kind.STD:
            # d(sqrt v) = dv / (2 sqrt v)
            tol = np.minimum(vtol / np.maximum(2.0 * b64[fin], 1e-300), np.sqrt(vtol))
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


def var_bound(cnt, var_pop, vmin, vmax, exact_in_f64=True):
    """Absolute VAR tolerance per group (module doc): VAR_EPS * n * (var +
    range^2), plus the int-to-double rounding term for integers beyond 2^53."""
    cnt = np.asarray(cnt, dtype=np.float64)
    rng = np.asarray(vmax, dtype=np.float64) - np.asarray(vmin, dtype=np.float64)
    tol = VAR_EPS * np.maximum(cnt, 1.0) * (np.asarray(var_pop, dtype=np.float64) + rng * rng)
    if not exact_in_f64:
        big = np.maximum(np.abs(np.asarray(vmin, dtype=np.float64)), np.abs(np.asarray(vmax, dtype=np.float64)))
        tol = tol + 4.0 * 2.0 ** -52 * big * np.abs(rng)
    return tol


def group_scales(keys: Sequence[HostCol], values: HostCol, null_policy, threads: int = 1) -> dict:
    """Per-group error scales in oracle group order, computed with the oracle
    itself: sum|x|, sum x^2, count, and the VAR bound var_bound() of the
    group's population variance and range."""
    vals = values.values if values.dict_keys is None else values.dict_keys.values[values.values]
    x = vals.astype(np.float64)
    absx = HostCol(np.abs(x), values.valid)
    sq = HostCol(x * x, values.valid)
    xc = HostCol(x, values.valid)
    r = orc.groupby(keys, [(absx, [(Kind.SUM, 0), (Kind.COUNT_VALID, 0)]), (sq, [(Kind.SUM, 0)]),
                           (xc, [(Kind.VARIANCE, 0), (Kind.MIN, 0), (Kind.MAX, 0)])], null_policy, threads)
    # the oracle is deterministic: same first-occurrence group order as the checked call
    f = lambda a: np.nan_to_num(np.asarray(a, dtype=np.float64), nan=0.0, posinf=0.0, neginf=0.0)
    cnt = np.asarray(r["results"][0][1][1], dtype=np.float64)
    exact = vals.dtype.kind == "f" or (len(vals) == 0 or float(np.max(np.abs(x))) <= 2.0 ** 53)
    vb = var_bound(cnt, f(r["results"][2][0][1]), f(r["results"][2][1][1]), f(r["results"][2][2][1]), exact)
    return {"abs": f(r["results"][0][0][1]), "cnt": cnt, "sq": f(r["results"][1][0][1]), "var": vb}


def sorted_group_scales(key: np.ndarray, x: np.ndarray, valid: Optional[np.ndarray]) -> dict:
    """The tolerance scales of group_scales() computed with numpy for one key
    column without nulls, for the groups in ascending key order (for inputs
    too large for the oracle to run a second time): sum|x|, count, and the
    VAR bound of each group's population variance and range."""
    order = np.argsort(key, kind="stable")
    ks = key[order]
    xs = x[order].astype(np.float64)
    vs = np.ones(len(xs), dtype=bool) if valid is None else np.asarray(valid, dtype=bool)[order]
    del order
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]]) if len(ks) else np.zeros(0, np.int64)
    del ks
    lengths = np.diff(np.r_[starts, len(xs)])
    cnt = np.add.reduceat(vs.astype(np.int64), starts).astype(np.float64)
    xz = np.where(vs, xs, 0.0)
    absx = np.add.reduceat(np.abs(xz), starts)
    mean = np.add.reduceat(xz, starts) / np.maximum(cnt, 1.0)
    d = np.where(vs, xs - np.repeat(mean, lengths), 0.0)
    var = np.add.reduceat(d * d, starts) / np.maximum(cnt, 1.0)
    del d
    mn = np.minimum.reduceat(np.where(vs, xs, np.inf), starts)
    mx = np.maximum.reduceat(np.where(vs, xs, -np.inf), starts)
    empty = cnt == 0
    mn[empty] = 0.0
    mx[empty] = 0.0
    exact = x.dtype.kind == "f" or (len(x) == 0 or float(np.max(np.abs(xs))) <= 2.0 ** 53)
    return {"abs": absx, "cnt": cnt, "var": var_bound(cnt, var, mn, mx, exact)}


def assert_parity(keys: Sequence[HostCol], requests, null_policy=NullPolicy.EXCLUDE, strategy=None, gpu=None,
                  threads: int = 1, keys_are_sorted=False):
    """Full parity check of libgbx against the oracle on the same inputs.
    With keys_are_sorted the groups are the reference's sort-path groups
    (oracle/presorted.py) and must come out in its order."""
    struct_keys = any(k.type_id == TypeId.STRUCT for k in keys)
    if keys_are_sorted:
        want = orc_sorted.groupby(keys, requests, null_policy, threads)
    elif struct_keys:
        want = orc_structs.groupby(keys, requests, null_policy, threads)
    else:
        want = orc.groupby(keys, requests, null_policy, threads)
    got = gpu if gpu is not None else run_gpu(keys, requests, null_policy, strategy, keys_are_sorted)
    assert got["num_groups"] == want["num_groups"], f"groups {got['num_groups']} != {want['num_groups']}"
    got_keys, want_keys = got["keys"], want["keys"]
    if struct_keys:
        # leaf by leaf (oracle/structs.py)
        got_keys = [leaf for k in got["keys"] for leaf in orc_structs.flatten_output(*k)]
        if keys_are_sorted:
            want_keys = [leaf for k in want["keys"] for leaf in orc_structs.flatten_output(*k)]
    if keys_are_sorted:
        go = wo = np.arange(want["num_groups"])
    else:
        go = sort_order(got_keys)
        wo = sort_order(want_keys)
    compare_keys(got_keys, want_keys, go, wo)
    for q, (vals, aggs) in enumerate(requests):
        vt = vals.dict_keys.type_id if vals.dict_keys is not None else vals.type_id
        is_float = vt in (TypeId.FLOAT32, TypeId.FLOAT64)
        sc = None
        for k, agg in enumerate(aggs):
            kind = Kind(agg[0])
            extra = agg[2] if len(agg) > 2 else {}
            ctx = f"request {q} agg {kind.name}"
            s = v = None
            if kind in (Kind.VARIANCE, Kind.STD, Kind.M2) or (
                    is_float and kind in (Kind.SUM, Kind.MEAN, Kind.SUM_OF_SQUARES)):
                if sc is None and keys_are_sorted:
                    # the scales of the label groups, in output order
                    sc = group_scales([want["label"]], vals, NullPolicy.EXCLUDE, threads)
                    sc = {name: a[want["perm"]] for name, a in sc.items()}
                elif sc is None and struct_keys:
                    sc = group_scales(want["enc"], vals, NullPolicy.EXCLUDE, threads)
                elif sc is None:
                    sc = group_scales(keys, vals, null_policy, threads)
                if kind == Kind.SUM:
                    s = sc["abs"]
                elif kind == Kind.MEAN:
                    s = sc["abs"] / np.maximum(sc["cnt"], 1)
                elif kind == Kind.SUM_OF_SQUARES:
                    s = sc["sq"]
                elif kind == Kind.M2:
                    # M2 = (n - ddof) VAR: the VAR bound times the group's count
                    v = sc["var"] * np.maximum(sc["cnt"], 1)
                else:
                    v = sc["var"]
            # QUANTILE: num_quantiles result rows per group
            nq = len(extra.get("quantiles", ())) if kind == Kind.QUANTILE else 1
            # MEDIAN / QUANTILE: the same double operations in the same order
            # as the oracle, so equal results
            compare_values(kind, got["results"][q][k], want["results"][q][k], rows_of_groups(go, nq),
                           rows_of_groups(wo, nq), s, v, ctx, exact=kind in (Kind.MEDIAN, Kind.QUANTILE))
    return got, want
