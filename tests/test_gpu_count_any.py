"""COUNT_VALID / COUNT_ALL over value columns the other kinds cannot read
(STRING, STRUCT): the reference answers them on its hash path (COUNT has a
size_type target whatever the values, hash/groupby.cu:73-84); here through
the C ABI against the oracle given an INT8 column with the same validity
(a count depends on nothing else).  Kinds other than COUNT (and MIN / MAX
of strings, tests/test_gpu_string_values.py) stay GBX_ERR_UNSUPPORTED."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from cudf_b200._lib import UnsupportedError
from oracle import oracle as orc
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

COUNTS = [(Kind.COUNT_VALID, 0), (Kind.COUNT_ALL, 0)]


def _values(rng, n):
    words = np.array(["", "a", "bb", "año"], dtype=object)
    valid = rng.random(n) >= 0.2
    s = HostCol(list(words[rng.integers(0, len(words), n)]), valid, type_id=TypeId.STRING)
    sv = rng.random(n) >= 0.3
    st = HostCol(None, sv, type_id=TypeId.STRUCT, children=[HostCol(rng.integers(0, 5, n).astype(np.int32))])
    return (s, valid), (st, sv)


@pytest.mark.parametrize("policy", [NullPolicy.EXCLUDE, NullPolicy.INCLUDE], ids=lambda p: p.name)
def test_counts_of_string_and_struct_values(policy):
    rng = np.random.default_rng(91)
    n = 200_000
    k = rng.integers(0, 5_000, n).astype(np.int64)
    kv = rng.random(n) >= 0.05
    (s, svalid), (st, stvalid) = _values(rng, n)
    got = T.run_gpu([HostCol(k, kv)], [(s, COUNTS), (st, COUNTS)], policy)
    stand_in = [(HostCol(np.zeros(n, np.int8), svalid), COUNTS), (HostCol(np.zeros(n, np.int8), stvalid), COUNTS)]
    want = orc.groupby([HostCol(k, kv)], stand_in, policy)
    go, wo = T.sort_order(got["keys"]), T.sort_order(want["keys"])
    T.compare_keys(got["keys"], want["keys"], go, wo)
    for q in range(2):
        for j in range(2):
            T.compare_values(COUNTS[j][0], got["results"][q][j], want["results"][q][j], go, wo)


def test_sliced_string_values_and_other_kinds_refused():
    rng = np.random.default_rng(92)
    n = 10_000
    k = rng.integers(0, 50, n).astype(np.int32)
    (s, svalid), _ = _values(rng, n)
    sl = HostCol(s.values, s.valid, type_id=TypeId.STRING, offset=100, size=5_000)
    ks = HostCol(k, offset=100, size=5_000)
    got = T.run_gpu([ks], [(sl, COUNTS)])
    want = orc.groupby([ks], [(HostCol(np.zeros(n, np.int8), svalid, offset=100, size=5_000), COUNTS)])
    go, wo = T.sort_order(got["keys"]), T.sort_order(want["keys"])
    for j in range(2):
        T.compare_values(COUNTS[j][0], got["results"][0][j], want["results"][0][j], go, wo)
    with pytest.raises(UnsupportedError):
        T.run_gpu([HostCol(k)], [(s, [(Kind.SUM, 0)])])
