"""The oracle's sort-path kinds (MEDIAN, QUANTILE, NUNIQUE, NTH_ELEMENT, M2)
against independent CPU computations (numpy / pandas) on seeded random
inputs, so that the oracle the GPU parity tests rely on is pinned by more than
the reference's small known-answer vectors."""
from __future__ import annotations

import numpy as np
import pandas as pd
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle import oracle as orc
from oracle.oracle import HostCol
from tests import gbx_testing as T


def _groups(n, card, seed, dtype=np.float64, null_frac=0.2, nan_frac=0.0):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, card, n).astype(np.int32)
    if np.dtype(dtype).kind == "f":
        v = rng.normal(0, 100, n).astype(dtype)
        v[rng.random(n) < nan_frac] = np.nan
    else:
        v = rng.integers(-50, 50, n).astype(dtype)
    valid = rng.random(n) >= null_frac
    return k, v, valid


def _oracle_by_key(k, v, valid, aggs):
    r = orc.groupby([HostCol(k)], [(HostCol(v, valid), aggs)])
    keys = r["keys"][0][1]
    return keys, r["results"][0]


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float32, np.float64])
def test_quantiles_match_numpy(dtype):
    k, v, valid = _groups(5000, 40, 1, dtype)
    qs = [0.0, 0.1, 0.5, 0.77, 1.0]
    keys, res = _oracle_by_key(k, v, valid, [(Kind.MEDIAN, 0), (Kind.QUANTILE, 0, {"quantiles": qs}),
                                             (Kind.QUANTILE, 0, {"quantiles": [0.3], "interpolation": 1}),
                                             (Kind.QUANTILE, 0, {"quantiles": [0.3], "interpolation": 2})])
    nq = len(qs)
    for g, key in enumerate(keys):
        x = np.sort(v[(k == key) & valid].astype(np.float64))
        if len(x) == 0:
            assert not res[0][2][g]
            continue
        assert res[0][1][g] == pytest.approx(np.quantile(x, 0.5), rel=1e-12, abs=1e-12)
        want = np.quantile(x, qs)  # numpy's default: linear interpolation
        assert np.allclose(res[1][1][g * nq:(g + 1) * nq], want, rtol=1e-12, atol=1e-12)
        assert res[2][1][g] == np.quantile(x, 0.3, method="lower")
        assert res[3][1][g] == np.quantile(x, 0.3, method="higher")


def test_quantiles_sort_nan_last():
    """NaN orders after every number (values are sorted as the reference's
    sort does): a group's upper quantiles are NaN once NaN reaches them."""
    k = np.array([1, 1, 1, 1, 2, 2], np.int32)
    v = np.array([np.nan, 3.0, 1.0, 2.0, -0.0, 0.0])
    keys, res = _oracle_by_key(k, v, None, [(Kind.QUANTILE, 0, {"quantiles": [0.0, 0.5, 1.0], "interpolation": 1})])
    g1 = int(np.nonzero(keys == 1)[0][0])
    got = res[0][1][3 * g1:3 * g1 + 3]
    assert got[0] == 1.0 and got[1] == 2.0 and np.isnan(got[2])


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE])
def test_nunique_matches_pandas(policy):
    k, v, valid = _groups(4000, 30, 2, np.float64, nan_frac=0.05)
    v = np.round(v / 40.0) * 40.0  # repeated values
    v[::97] = -0.0                 # -0.0 and +0.0 are one value
    keys, res = _oracle_by_key(k, v, valid, [(Kind.NUNIQUE, 0, {"null_policy": policy})])
    # pd.unique keeps NaN as one value (NaNs equal) and -0.0 / +0.0 apart,
    # so zeros are folded first
    for g, key in enumerate(keys):
        m = k == key
        vals = v[m & valid]
        want = len(pd.unique(np.where(vals == 0, 0.0, vals)))
        if policy == NullPolicy.INCLUDE and (~valid[m]).any():
            want += 1
        assert res[0][1][g] == want, key


@pytest.mark.parametrize("n", [0, 1, 2, -1, -3])
@pytest.mark.parametrize("policy", [NullPolicy.INCLUDE, NullPolicy.EXCLUDE])
def test_nth_element_matches_pandas(n, policy):
    k, v, valid = _groups(3000, 50, 3, np.int64, null_frac=0.3)
    keys, res = _oracle_by_key(k, v, valid, [(Kind.NTH_ELEMENT, n, {"null_policy": policy})])
    _, got, got_valid = res[0]
    df = pd.DataFrame({"k": k, "v": pd.array(np.where(valid, v, 0), dtype="Int64"), "ok": valid})
    df.loc[~df.ok, "v"] = pd.NA
    src = df if policy == NullPolicy.INCLUDE else df[df.ok]
    want = src.groupby("k")["v"].nth(n)
    want = dict(zip(src.loc[want.index, "k"], want))
    gv = np.ones(len(keys), bool) if got_valid is None else got_valid
    for g, key in enumerate(keys):
        w = want.get(key, pd.NA)
        if w is pd.NA:
            assert not gv[g], key
        else:
            assert gv[g] and got[g] == w, key


def test_m2_matches_two_pass_numpy():
    k, v, valid = _groups(6000, 60, 4, np.float64)
    keys, res = _oracle_by_key(k, v, valid, [(Kind.M2, 0)])
    for g, key in enumerate(keys):
        x = v[(k == key) & valid]
        if len(x) == 0:
            assert not res[0][2][g]
            continue
        assert res[0][1][g] == pytest.approx(float(((x - x.mean()) ** 2).sum()), rel=1e-12, abs=1e-9)


def test_quantile_result_rows_per_group():
    k = np.array([2, 1, 2, 1, 2], np.int32)
    v = np.array([5, 1, 7, 3, 6], np.int32)
    r = orc.groupby([HostCol(k)], [(HostCol(v), [(Kind.QUANTILE, 0, {"quantiles": [0.0, 0.5, 1.0]})])])
    tid, vals, valid = r["results"][0][0]
    assert tid == TypeId.FLOAT64 and len(vals) == 3 * r["num_groups"]
    order = T.rows_of_groups(T.sort_order(r["keys"]), 3)
    assert list(vals[order]) == [1.0, 2.0, 3.0, 5.0, 6.0, 7.0]
