"""GPU parity of STRUCT key columns: the reference gtests' known answers
(tests/golden/struct_kats.py) and seeded inputs against the struct-key oracle
(oracle/structs.py), through the C ABI.  Keys are compared leaf by leaf (a
struct's validity, then its members', each carrying the enclosing structs'
nulls) after a sort by key; tolerances are those of tests/gbx_testing.py."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, Strategy, TypeId
from oracle import structs as S
from oracle.oracle import HostCol
from tests import gbx_testing as T
from tests.test_struct_keys import CASES, build, check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_gpu_matches_struct_kat(case):
    keys, reqs = build(case)
    got = T.run_gpu(keys, reqs, NullPolicy.INCLUDE)
    leaves = [leaf for k in got["keys"] for leaf in S.flatten_output(*k)]
    check(leaves, got["results"][0][0], case)


def _struct(rng, n, null_rate=0.1, member_null=0.1, card=50):
    a = rng.integers(0, card, n).astype(np.int32)
    av = rng.random(n) >= member_null
    words = np.array(["", "x", "xy", "año", "₹1", "long-" * 5], dtype=object)
    s = list(words[rng.integers(0, len(words), n)])
    sv = rng.random(n) >= member_null
    f = rng.integers(-2, 3, n).astype(np.float64)
    f[rng.random(n) < 0.05] = np.nan
    f[f == 0] = np.where(rng.random(int((f == 0).sum())) < 0.5, -0.0, 0.0)
    members = [HostCol(a, av), HostCol(s, sv, type_id=TypeId.STRING), HostCol(f)]
    return HostCol(None, rng.random(n) >= null_rate, type_id=TypeId.STRUCT, children=members)


AGGS = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.COUNT_ALL, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0),
        (Kind.VARIANCE, 1), (Kind.ARGMIN, 0), (Kind.ARGMAX, 0), (Kind.MEDIAN, 0), (Kind.NUNIQUE, 0)]


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_struct_key_with_nulls_everywhere(policy):
    rng = np.random.default_rng(61)
    n = 60_000
    k = _struct(rng, n)
    v = rng.integers(-1000, 1000, n).astype(np.int64)
    vv = rng.random(n) >= 0.1
    T.assert_parity([k], [(HostCol(v, vv), AGGS)], policy)


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_struct_beside_plain_columns_and_nested(policy):
    rng = np.random.default_rng(62)
    n = 40_000
    inner = _struct(rng, n, card=6)
    b = rng.integers(0, 3, n).astype(np.int16)
    outer = HostCol(None, rng.random(n) >= 0.05, type_id=TypeId.STRUCT,
                    children=[inner, HostCol(b, rng.random(n) >= 0.05)])
    plain = rng.integers(0, 4, n).astype(np.int64)
    pv = rng.random(n) >= 0.05
    v = rng.normal(0, 1, n).astype(np.float32)
    T.assert_parity([HostCol(plain, pv), outer], [(HostCol(v), [(Kind.SUM, 0), (Kind.MEAN, 0), (Kind.MAX, 0)])],
                    policy)


@pytest.mark.parametrize("strategy", [Strategy.AUTO, Strategy.GLOBAL, Strategy.PARTITIONED, Strategy.WARP],
                         ids=lambda s: s.name)
def test_many_groups_every_strategy(strategy):
    rng = np.random.default_rng(63)
    n = 300_000
    k = _struct(rng, n, null_rate=0.01, member_null=0.01, card=50_000)
    v = rng.integers(0, 100, n).astype(np.int32)
    T.assert_parity([k], [(HostCol(v), [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.ARGMAX, 0)])], strategy=strategy)


def test_sliced_struct_and_all_null_structs():
    rng = np.random.default_rng(64)
    n = 5_000
    k = _struct(rng, n)
    v = HostCol(rng.integers(0, 9, n).astype(np.int32), offset=100, size=4_000)
    ks = HostCol(None, k.valid, type_id=TypeId.STRUCT, children=k.children, offset=100, size=4_000)
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        T.assert_parity([ks], [(v, [(Kind.SUM, 0), (Kind.ARGMIN, 0)])], policy)
    dead = HostCol(None, np.zeros(n, bool), type_id=TypeId.STRUCT, children=k.children)
    w = HostCol(np.ones(n, np.int32))
    for policy in (NullPolicy.EXCLUDE, NullPolicy.INCLUDE):
        got, _ = T.assert_parity([dead], [(w, [(Kind.SUM, 0)])], policy)
        assert got["num_groups"] == (0 if policy == NullPolicy.EXCLUDE else 1)


def test_sorted_struct_keys_group_as_runs():
    """keys_are_sorted with struct keys whose equal rows are adjacent: the
    runs are the groups, in row order."""
    rng = np.random.default_rng(65)
    n = 20_000
    a = np.sort(rng.integers(0, 300, n)).astype(np.int32)
    k = HostCol(None, None, type_id=TypeId.STRUCT, children=[HostCol(a), HostCol((a % 7).astype(np.int8))])
    v = HostCol(rng.integers(0, 50, n).astype(np.int64))
    got = T.run_gpu([k], [(v, [(Kind.SUM, 0)])], NullPolicy.INCLUDE, keys_are_sorted=True)
    want = S.groupby([k], [(v, [(Kind.SUM, 0)])], NullPolicy.INCLUDE)
    leaves = [leaf for kk in got["keys"] for leaf in S.flatten_output(*kk)]
    first = leaves[1][1]
    assert np.all(np.diff(first) > 0), "groups come out in row order"
    go, wo = T.sort_order(leaves), T.sort_order(want["keys"])
    T.compare_keys(leaves, want["keys"], go, wo)
    T.compare_values(Kind.SUM, got["results"][0][0], want["results"][0][0], go, wo)
