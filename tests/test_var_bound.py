"""The VAR/STD tolerance of the parity tests has teeth (CPU only).

The GPU's shifted one-pass moments are restated here in numpy (sum (x-K)^2
and sum (x-K) accumulated row by row, K the group's first value) and checked
against the oracle under the stated bound; two planted mistakes -- the naive
sum x^2 - n mean^2, and S1 derived from the plain sum as sum x - n K -- must
fail it on values with |mean| >> std.  The mistakes are planted in this CPU
restatement, never in the library.
"""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle import oracle as orc
from oracle.oracle import HostCol
from tests import gbx_testing as T


def _data(n=60_000, groups=120, offset=1e9, seed=17):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, groups, size=n).astype(np.int32)
    v = offset + rng.standard_normal(n)
    return k, v


def _per_group(keys_in_order, k, v, ddof, variant):
    """VAR per group (in the oracle's group order) by a sequential float64
    restatement of the kernels' arithmetic, or by a planted mistake."""
    out = np.empty(len(keys_in_order))
    for gi, key in enumerate(keys_in_order):
        x = v[k == key]
        n = len(x)
        K = x[0]
        if variant == "naive":
            s, q = 0.0, 0.0
            for xi in x:
                s += xi
                q += xi * xi
            m2 = max(q - n * (s / n) ** 2, 0.0)
        else:
            s, s1, s2 = 0.0, 0.0, 0.0
            for xi in x:
                d = xi - K
                s += xi
                s1 += d
                s2 += d * d
            S1 = s1 if variant == "shifted" else s - n * K
            m2 = max(s2 - S1 * (S1 / n), 0.0)
        out[gi] = m2 / (n - ddof)
    return out


@pytest.mark.parametrize("ddof", [0, 1])
def test_var_bound_accepts_shifted_and_rejects_cancelling_forms(ddof):
    k, v = _data()
    keys = [HostCol(k)]
    vals = HostCol(v)
    want = orc.groupby(keys, [(vals, [(Kind.VARIANCE, ddof), (Kind.STD, ddof)])], NullPolicy.EXCLUDE)
    gkeys = np.asarray(want["keys"][0][1])
    sc = T.group_scales(keys, vals, NullPolicy.EXCLUDE)
    order = np.arange(len(gkeys))
    wvar = want["results"][0][0]
    wstd = want["results"][0][1]

    def check(var, kind, wcol):
        got = (int(TypeId.FLOAT64), var if kind == Kind.VARIANCE else np.sqrt(var), None)
        T.compare_values(kind, got, wcol, order, order, None, sc["var"], ctx=kind.name)

    shifted = _per_group(gkeys, k, v, ddof, "shifted")
    check(shifted, Kind.VARIANCE, wvar)
    check(shifted, Kind.STD, wstd)
    for planted in ("naive", "derived_s1"):
        bad = _per_group(gkeys, k, v, ddof, planted)
        with pytest.raises(AssertionError, match="out of bound"):
            check(bad, Kind.VARIANCE, wvar)
        with pytest.raises(AssertionError, match="out of bound"):
            check(bad, Kind.STD, wstd)


def test_var_bound_scales_with_variance_not_mean():
    """The bound is of the order of n * 2^-52 * (var + range^2), so it stays
    small against the variance however large the mean."""
    k, v = _data(n=20_000, groups=40)
    sc = T.group_scales([HostCol(k)], HostCol(v), NullPolicy.EXCLUDE)
    want = orc.groupby([HostCol(k)], [(HostCol(v), [(Kind.VARIANCE, 0)])], NullPolicy.EXCLUDE)
    var = np.asarray(want["results"][0][0][1])
    assert np.all(sc["var"] < 1e-9 * var)


def test_sorted_group_scales_match_the_oracle_scales():
    """The numpy scales used by the full-size tests equal the oracle's."""
    rng = np.random.default_rng(5)
    n = 50_000
    k = rng.integers(0, 3_000, size=n).astype(np.int64)
    x = rng.standard_normal(n).astype(np.float32)
    valid = rng.random(n) >= 0.1
    sc = T.sorted_group_scales(k, x, valid)
    ref = T.group_scales([HostCol(k)], HostCol(x, valid), NullPolicy.EXCLUDE)
    keys = orc.groupby([HostCol(k)], [(HostCol(x, valid), [(Kind.COUNT_ALL, 0)])], NullPolicy.EXCLUDE)["keys"][0][1]
    order = np.argsort(keys)
    for name in ("abs", "cnt", "var"):
        np.testing.assert_allclose(sc[name], ref[name][order], rtol=1e-9, atol=1e-300)
