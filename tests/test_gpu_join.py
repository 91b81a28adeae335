"""GPU parity of gbx_hash_join (inner, left, full, left semi, left anti)
against the join oracle (oracle/join.py) through the C ABI: the reference
gtests' known answers (tests/golden/join_kats.py) and seeded inputs with
repeated keys, skew, STRING and STRUCT keys, NaN / signed-zero float keys and
nulls under both null equalities.  The gather maps are compared as sorted
sets of (left row, right row) pairs -- bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200 import Table
from cudf_b200 import join as J
from cudf_b200._abi import JoinKind, NullEquality, TypeId
from oracle import join as OJ
from oracle.oracle import HostCol
from tests import gbx_testing as T
from tests.test_join import CASES, keys_of

pytestmark = pytest.mark.gpu

NONE = -(2 ** 31)
KINDS = [JoinKind.INNER, JoinKind.LEFT, JoinKind.FULL, JoinKind.LEFT_SEMI, JoinKind.LEFT_ANTI]


def gpu_pairs(left, right, nulls, kind):
    lt = Table([T.device_column(k) for k in left])
    rt = Table([T.device_column(k) for k in right])
    fn = {JoinKind.INNER: J.inner_join, JoinKind.LEFT: J.left_join, JoinKind.FULL: J.full_join,
          JoinKind.LEFT_SEMI: J.left_semi_join, JoinKind.LEFT_ANTI: J.left_anti_join}[kind]
    out = fn(lt, rt, nulls)
    if kind in (JoinKind.LEFT_SEMI, JoinKind.LEFT_ANTI):
        li = out.to_numpy()[0]
        ri = np.full(len(li), NONE, dtype=np.int64)
    else:
        li, ri = out[0].to_numpy()[0], out[1].to_numpy()[0]
    pairs = [(None if a == NONE else int(a), None if b == NONE else int(b)) for a, b in zip(li, ri)]
    return sorted(pairs, key=lambda p: (-1 if p[0] is None else p[0], -1 if p[1] is None else p[1]))


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_gpu_matches_join_kat(case):
    got = gpu_pairs(keys_of(case["left"]), keys_of(case["right"]), case["nulls"], case["kind"])
    want = sorted(case["pairs"], key=lambda p: (-1 if p[0] is None else p[0], -1 if p[1] is None else p[1]))
    assert got == want


def _check(left, right, nulls, kind):
    got = gpu_pairs(left, right, nulls, kind)
    want = OJ.hash_join(left, right, nulls, kind)
    assert len(got) == len(want), f"{len(got)} pairs, expected {len(want)}"
    assert got == want


@pytest.mark.parametrize("kind", KINDS, ids=lambda k: k.name)
@pytest.mark.parametrize("nulls", [NullEquality.EQUAL, NullEquality.UNEQUAL], ids=lambda e: e.name)
def test_repeated_int_keys_with_nulls(kind, nulls):
    rng = np.random.default_rng(71)
    nl, nr = 20_000, 6_000
    a = rng.integers(0, 3_000, nl).astype(np.int64)
    b = rng.integers(0, 3_000, nr).astype(np.int64)
    b[:500] = 7  # one key repeated many times on the build side
    av = rng.random(nl) >= 0.05
    bv = rng.random(nr) >= 0.05
    _check([HostCol(a, av)], [HostCol(b, bv)], nulls, kind)


@pytest.mark.parametrize("kind", KINDS, ids=lambda k: k.name)
def test_string_and_int_keys(kind):
    rng = np.random.default_rng(72)
    words = np.array(["", "a", "ab", "año", "₹1", "x" * 33, "zz"], dtype=object)
    nl, nr = 8_000, 9_000  # the right side larger: an inner join builds the left
    ls = list(words[rng.integers(0, len(words), nl)])
    rs = list(words[rng.integers(0, len(words), nr)])
    li = rng.integers(0, 40, nl).astype(np.int32)
    ri = rng.integers(0, 40, nr).astype(np.int32)
    lsv = rng.random(nl) >= 0.1
    left = [HostCol(ls, lsv, type_id=TypeId.STRING), HostCol(li)]
    right = [HostCol(rs, type_id=TypeId.STRING), HostCol(ri)]
    for nulls in (NullEquality.EQUAL, NullEquality.UNEQUAL):
        _check(left, right, nulls, kind)


@pytest.mark.parametrize("kind", [JoinKind.INNER, JoinKind.FULL, JoinKind.LEFT_ANTI], ids=lambda k: k.name)
def test_struct_and_float_keys(kind):
    rng = np.random.default_rng(73)

    def side(n):
        a = rng.integers(0, 20, n).astype(np.int32)
        av = rng.random(n) >= 0.1
        f = rng.integers(-2, 3, n).astype(np.float64)
        f[rng.random(n) < 0.1] = np.nan
        f[f == 0] = np.where(rng.random(int((f == 0).sum())) < 0.5, -0.0, 0.0)
        s = HostCol(None, rng.random(n) >= 0.1, type_id=TypeId.STRUCT, children=[HostCol(a, av), HostCol(f)])
        return [s, HostCol(rng.integers(0, 3, n).astype(np.int8))]

    left, right = side(5_000), side(4_000)
    for nulls in (NullEquality.EQUAL, NullEquality.UNEQUAL):
        _check(left, right, nulls, kind)


def test_empty_sides_and_no_matches():
    e = [HostCol(np.zeros(0, np.int32))]
    x = [HostCol(np.arange(5, dtype=np.int32))]
    y = [HostCol(np.arange(100, 103, dtype=np.int32))]
    for kind in KINDS:
        _check(e, x, NullEquality.EQUAL, kind)
        _check(x, e, NullEquality.EQUAL, kind)
        _check(x, y, NullEquality.EQUAL, kind)


def test_large_skewed_inner_join():
    """Many probe rows on a few hot keys: the output is large, each probe row
    writes its key's run of build rows."""
    rng = np.random.default_rng(74)
    nl, nr = 200_000, 500
    a = rng.integers(0, 10, nl).astype(np.int32)
    b = rng.integers(0, 10, nr).astype(np.int32)
    li, ri = J.inner_join(Table([T.device_column(HostCol(a))]), Table([T.device_column(HostCol(b))]))
    ga, gb = li.to_numpy()[0].astype(np.int64), ri.to_numpy()[0].astype(np.int64)
    cnt = np.bincount(b, minlength=10)
    assert len(ga) == int(cnt[a].sum())
    assert np.array_equal(a[ga], b[gb])
    # every (left, right) pair of equal keys appears exactly once
    assert len(np.unique(ga * nr + gb)) == len(ga)
