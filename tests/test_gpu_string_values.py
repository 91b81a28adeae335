"""MIN / MAX of STRING values (libcudf computes them on its sort path) through
the C ABI: the reference gtests' known answers (min_tests.cpp /
max_tests.cpp string cases) and seeded inputs against a Python restatement
(per group the least / greatest valid string in byte order, null where a
group has no valid value), with COUNT and numeric requests in the same call,
null keys under both policies, STRUCT keys and sliced columns."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu


def _by_key(got, q):
    """{key: (min, max, count)} from a result whose request q holds MIN, MAX,
    COUNT_VALID (key None: the null key)."""
    kt, kv, kvalid = got["keys"][0]
    n = len(kv)
    kvalid = np.ones(n, bool) if kvalid is None else kvalid
    (_, mn, mnv), (_, mx, mxv), (_, cnt, _) = got["results"][q][:3]
    mnv = np.ones(n, bool) if mnv is None else mnv
    mxv = np.ones(n, bool) if mxv is None else mxv
    out = {}
    for i in range(n):
        key = int(kv[i]) if kvalid[i] else None
        out[key] = (mn[i] if mnv[i] else None, mx[i] if mxv[i] else None, int(cnt[i]))
    return out


def _expect(keys, kvalid, vals, vvalid, policy):
    out = {}
    for k, kok, v, vok in zip(keys, kvalid, vals, vvalid):
        if not kok and policy == NullPolicy.EXCLUDE:
            continue
        key = int(k) if kok else None
        mn, mx, c = out.get(key, (None, None, 0))
        if vok:
            b = v.encode("utf-8")
            mn = v if mn is None or b < mn.encode("utf-8") else mn
            mx = v if mx is None or b > mx.encode("utf-8") else mx
            c += 1
        out[key] = (mn, mx, c)
    return out


AGGS = [(Kind.MIN, 0), (Kind.MAX, 0), (Kind.COUNT_VALID, 0)]


def test_reference_basic_and_zero_valid():
    """min_tests.cpp:134-163, max_tests.cpp:134-148."""
    k = HostCol(np.array([1, 2, 3, 1, 2, 2, 1, 3, 3, 2], np.int32))
    v = HostCol(["año", "bit", "₹1", "aaa", "zit", "bat", "aaa", "$1", "₹1", "wut"], type_id=TypeId.STRING)
    got = _by_key(T.run_gpu([k], [(v, AGGS)]), 0)
    assert {key: got[key][:2] for key in got} == {1: ("aaa", "año"), 2: ("bat", "zit"), 3: ("$1", "₹1")}
    k1 = HostCol(np.array([1, 1, 1], np.int32))
    v1 = HostCol(["año", "bit", "₹1"], np.zeros(3, bool), type_id=TypeId.STRING)
    assert _by_key(T.run_gpu([k1], [(v1, AGGS)]), 0) == {1: (None, None, 0)}


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_strings_with_numeric_requests(policy):
    rng = np.random.default_rng(101)
    n = 150_000
    words = np.array(["", "a", "aa", "ab", "b", "año", "ano", "₹1", "z" * 30, "zz"], dtype=object)
    k = rng.integers(0, 3_000, n).astype(np.int64)
    kv = rng.random(n) >= 0.05
    s = list(words[rng.integers(0, len(words), n)])
    sv = rng.random(n) >= 0.3
    x = rng.integers(-100, 100, n).astype(np.int32)
    got = T.run_gpu([HostCol(k, kv)], [(HostCol(x), [(Kind.SUM, 0)]),
                                      (HostCol(s, sv, type_id=TypeId.STRING), AGGS)], policy)
    assert _by_key(got, 1) == _expect(k, kv, s, sv, policy)
    kt, keys, kvalid = got["keys"][0]
    kvalid = np.ones(len(keys), bool) if kvalid is None else kvalid
    want = {}
    for kk, ok, xx in zip(k, kv, x):
        if ok or policy == NullPolicy.INCLUDE:
            key = int(kk) if ok else None
            want[key] = want.get(key, 0) + int(xx)
    sums = got["results"][0][0][1]
    assert {(int(a) if ok else None): int(b) for a, ok, b in zip(keys, kvalid, sums)} == want


def test_only_string_extremes_struct_keys_and_slices():
    rng = np.random.default_rng(102)
    n = 20_000
    a = rng.integers(0, 50, n).astype(np.int32)
    st = HostCol(None, None, type_id=TypeId.STRUCT, children=[HostCol(a)])
    words = np.array(["q", "r", "s", "ŝ"], dtype=object)
    s = list(words[rng.integers(0, len(words), n)])
    got = T.run_gpu([st], [(HostCol(s, type_id=TypeId.STRING), [(Kind.MAX, 0)])])
    members = got["keys"][0][1]
    gk = members[0][1]
    want = {}
    for aa, ss in zip(a, s):
        want[int(aa)] = max(want.get(int(aa), ss), ss, key=lambda t: t.encode("utf-8"))
    mx = got["results"][0][0][1]
    assert {int(x): y for x, y in zip(gk, mx)} == want
    ks = HostCol(a, offset=100, size=5_000)
    vs = HostCol(s, type_id=TypeId.STRING, offset=100, size=5_000)
    got = T.run_gpu([ks], [(vs, AGGS)])
    assert _by_key(got, 0) == _expect(a[100:5100], np.ones(5000, bool), s[100:5100], np.ones(5000, bool),
                                      NullPolicy.EXCLUDE)
