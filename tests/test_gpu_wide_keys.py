"""GPU parity of the groupby over keys that do not pack into two 64-bit
words -- STRING key columns and fixed-width keys beyond 128 bits with their
null bits -- against the oracle, through the C ABI: null policies, nulls in
keys and values, NaN / signed-zero floats, empty strings, non-ASCII text and
several aggregations, at sizes from a few rows to millions."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

AGGS = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.COUNT_ALL, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0),
        (Kind.VARIANCE, 1)]


def _words(rng, n, card, null_frac=0.0):
    pool = ["", "a", "ab", "año", "₹1", "x" * 40, "longer key text", "Zz"] + [f"k{i:05d}" for i in range(card)]
    pool = pool[:max(card, 1)]
    vals = [pool[i] for i in rng.integers(0, len(pool), n)]
    if null_frac:
        for i in np.nonzero(rng.random(n) < null_frac)[0]:
            vals[i] = None
    return vals


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
@pytest.mark.parametrize("n,card", [(1_000, 20), (200_000, 5_000), (2_000_000, 300)])
def test_string_keys(policy, n, card):
    rng = np.random.default_rng(n + card)
    k = HostCol(_words(rng, n, card, 0.05), type_id=TypeId.STRING)
    v = rng.normal(0, 10, n)
    vv = rng.random(n) >= 0.1
    T.assert_parity([k], [(HostCol(v, vv), AGGS)], policy, threads=8 if n > 100_000 else 1)


def test_string_and_int_keys_with_sort_kinds():
    rng = np.random.default_rng(3)
    n = 100_000
    s = HostCol(_words(rng, n, 50, 0.02), type_id=TypeId.STRING)
    i = HostCol(rng.integers(0, 4, n).astype(np.int16), rng.random(n) >= 0.03)
    v = rng.integers(-100, 100, n).astype(np.int32)
    aggs = AGGS + [(Kind.MEDIAN, 0), (Kind.NUNIQUE, 0), (Kind.NTH_ELEMENT, 1, {"null_policy": NullPolicy.INCLUDE})]
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([s, i], [(HostCol(v), aggs)], policy)


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_keys_beyond_128_bits(policy):
    """Three int64 columns (192 bits); two nullable int64 and a float64
    (192 value bits and three null bits)."""
    rng = np.random.default_rng(4)
    n = 300_000
    a = rng.integers(0, 30, n).astype(np.int64)
    b = rng.integers(-5, 5, n).astype(np.int64) * (1 << 40)
    c = rng.integers(0, 3, n).astype(np.int64) - 1  # includes the all-ones word -1
    v = rng.normal(size=n)
    T.assert_parity([HostCol(a), HostCol(b), HostCol(c)], [(HostCol(v), AGGS)], policy)
    f = rng.choice([0.5, -0.0, 0.0, np.nan, 2.5], n)
    T.assert_parity([HostCol(a, rng.random(n) >= 0.05), HostCol(b, rng.random(n) >= 0.05), HostCol(f)],
                    [(HostCol(v), AGGS)], policy)


def test_empty_and_all_null_string_keys():
    T.assert_parity([HostCol([], type_id=TypeId.STRING)], [(HostCol(np.zeros(0)), AGGS)])
    k = HostCol([None, None, None], type_id=TypeId.STRING)
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([k], [(HostCol(np.array([1.0, 2.0, 3.0])), AGGS)], policy)
