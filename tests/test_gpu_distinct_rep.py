"""GPU parity of distinct_count / distinct_indices over STRING and STRUCT
keys (the representative-row path) with the oracle: the reference gtests'
known answers, then seeded inputs with nulls at every level, NaNs and signed
zeros, under both null and NaN equalities and every keep option.  Kept rows
are compared exactly for KEEP_FIRST / KEEP_LAST / KEEP_NONE, and as one row
per class for KEEP_ANY."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200 import Table
from cudf_b200 import stream_compaction as sc
from cudf_b200._abi import DuplicateKeep, NanEquality, NullEquality, TypeId
from oracle import distinct as od
from oracle.oracle import HostCol
from tests import gbx_testing as T
from tests.golden import distinct_kats as K
from tests.test_distinct_rep import classes_kept_once, leaf_cols, spec_host

pytestmark = pytest.mark.gpu


def dev(keys):
    return Table([T.device_column(k) for k in keys])


def test_string_key_column_kat():
    specs, want = K.STRING_KEY_COLUMN
    keys = [spec_host(s) for s in specs]
    t = dev(keys)
    for keep, rows in want.items():
        got = np.sort(sc.distinct_indices(t, DuplicateKeep(keep)).to_numpy()[0])
        assert list(got) == rows, keep
    assert sc.distinct_count(t) == 5


def test_structs_of_structs_kat():
    specs, want = K.STRUCTS_OF_STRUCTS
    t = dev([spec_host(s) for s in specs])
    eq = sc.distinct_indices(t, DuplicateKeep.KEEP_ANY, NullEquality.EQUAL).to_numpy()[0]
    uneq = sc.distinct_indices(t, DuplicateKeep.KEEP_ANY, NullEquality.UNEQUAL).to_numpy()[0]
    assert classes_kept_once(eq, want["equal"])
    assert classes_kept_once(uneq, want["unequal"])
    assert sc.distinct_count(t, NullEquality.EQUAL) == 6
    assert sc.distinct_count(t, NullEquality.UNEQUAL) == 8


def _keys(rng, n):
    words = np.array(["", "a", "ab", "año", "x" * 20], dtype=object)
    s = HostCol(list(words[rng.integers(0, len(words), n)]), rng.random(n) >= 0.1, type_id=TypeId.STRING)
    f = rng.integers(-1, 2, n).astype(np.float32)
    f[rng.random(n) < 0.1] = np.nan
    f[f == 0] = np.where(rng.random(int((f == 0).sum())) < 0.5, -0.0, 0.0)
    a = rng.integers(0, 3, n).astype(np.int16)
    st = HostCol(None, rng.random(n) >= 0.1, type_id=TypeId.STRUCT,
                 children=[HostCol(a, rng.random(n) >= 0.1), HostCol(f)])
    return [s, st]


@pytest.mark.parametrize("keep", list(DuplicateKeep), ids=lambda k: k.name)
@pytest.mark.parametrize("nulls", [True, False], ids=["nulls_equal", "nulls_unequal"])
@pytest.mark.parametrize("nans", [True, False], ids=["nans_equal", "nans_unequal"])
def test_string_and_struct_keys(keep, nulls, nans):
    rng = np.random.default_rng(81)
    n = 30_000
    keys = _keys(rng, n)
    got = np.sort(sc.distinct_indices(dev(keys), keep, NullEquality.EQUAL if nulls else NullEquality.UNEQUAL,
                                      NanEquality.ALL_EQUAL if nans else NanEquality.UNEQUAL).to_numpy()[0])
    cols = leaf_cols(keys)
    if keep == DuplicateKeep.KEEP_ANY:
        rk = od.row_keys(cols, nulls, nans)
        classes = {}
        for r, k in enumerate(rk):
            classes.setdefault(k, []).append(r)
        assert classes_kept_once(got, list(classes.values()))
    else:
        want = od.distinct_indices(cols, int(keep), nulls, nans)
        assert np.array_equal(got, want)


def test_counts_and_empty():
    rng = np.random.default_rng(82)
    keys = _keys(rng, 10_000)
    cols = leaf_cols(keys)
    for nulls in (True, False):
        assert sc.distinct_count(dev(keys), NullEquality.EQUAL if nulls else NullEquality.UNEQUAL) == \
            od.distinct_count(cols, nulls)
    e = [HostCol([], type_id=TypeId.STRING)]
    assert sc.distinct_count(dev(e)) == 0
    assert len(sc.distinct_indices(dev(e)).to_numpy()[0]) == 0


def test_distinct_table_with_string_and_struct_columns():
    """cudf::distinct over a STRING key: the kept rows of every column,
    gathered (distinct_tests.cpp:80-123 inputs, KEEP_FIRST)."""
    from cudf_b200 import Column

    keys = Column.from_strings(["all", "new", "new", "all", None, "the", "strings"])
    col = Column.from_numpy(np.array([0, 1, 2, 3, 4, 5, 6], np.int32), np.array([1, 0, 1, 1, 1, 1, 1], bool))
    st = Column.struct([col], np.array([1, 1, 1, 0, 1, 1, 1], bool))
    out = sc.distinct(Table([col, keys, st]), [1], DuplicateKeep.KEEP_FIRST)
    vals, valid = out[0].to_numpy()
    kv, kvalid = out[1].to_numpy()
    order = np.argsort(vals)
    assert list(vals[order]) == [0, 1, 4, 5, 6]
    assert list(kv[order]) == ["all", "new", "", "the", "strings"]
    assert list(kvalid[order]) == [True, True, False, True, True]
    members, svalid = out[2].to_numpy()
    assert list(members[0][0][order]) == [0, 1, 4, 5, 6]
