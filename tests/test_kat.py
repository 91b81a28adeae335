"""Known-answer tests: the reference gtests' vectors (tests/golden/reference_kats.py)
checked against the oracle (CPU) and against libgbx (GPU), sorted by key as
the reference harness does (cpp/tests/groupby/groupby_test_util.cpp:89-96).
Cases with sorted::YES keys go through oracle/presorted.py and libgbx's
keys_are_sorted path."""
from __future__ import annotations

import numpy as np
import pytest

from cudf_b200._abi import Kind, TypeId
from cudf_b200.column import storage_dtype
from oracle import oracle as orc
from oracle import presorted as orc_sorted
from oracle.oracle import HostCol
from tests import gbx_testing as T
from tests.golden import reference_kats as KAT

CASES = KAT.cases()


def _host(vals, valid, tid, scale=0, as_dict=False, offset=0, size=None):
    tid = TypeId(tid)
    if tid == TypeId.STRING:
        return HostCol(list(vals), None if valid is None else np.array(valid, bool), type_id=tid, offset=offset,
                       size=size)
    if tid == TypeId.BOOL8:
        arr = np.array([bool(v) for v in vals], dtype=np.uint8)
    else:
        arr = np.array(vals, dtype=storage_dtype(tid)) if len(vals) else np.zeros(0, storage_dtype(tid))
    vm = None if valid is None else np.array(valid, dtype=bool)
    if as_dict:
        uniq, idx = np.unique(arr, return_inverse=True)
        keys = HostCol(uniq, None, type_id=tid, scale=scale)
        return HostCol(idx.astype(np.int32), vm, dict_keys=keys, offset=offset, size=size)
    return HostCol(arr, vm, type_id=tid, scale=scale, offset=offset, size=size)


def build(case):
    if case["key_dict"]:
        placeholder = HostCol(np.arange(3, dtype=np.int32))  # contents never read on the key path
        keys = HostCol(np.array(case["keys"], dtype=np.int32), None if case["key_valid"] is None
                       else np.array(case["key_valid"], bool), dict_keys=placeholder)
    else:
        keys = _host(case["keys"], case["key_valid"], case["key_type"], offset=case["offset"], size=case["size"])
    vals = _host(case["values"], case["value_valid"], case["value_type"], case.get("value_scale", 0),
                 as_dict=case["value_dict"], offset=case["offset"], size=case["size"])
    return [keys], [(vals, [(case["kind"], case["ddof"], case["extra"])])]


def expected(case):
    kt = TypeId.INT32 if case["key_dict"] else TypeId(case["key_type"])
    if kt == TypeId.STRING:
        ek = np.array(case["expect_keys"], dtype=object)
    else:
        ek = np.array(case["expect_keys"], dtype=storage_dtype(kt)) if case["expect_keys"] else np.zeros(0, storage_dtype(kt))
    ekv = None if case["expect_key_valid"] is None else np.array(case["expect_key_valid"], bool)
    rt = TypeId(case["result_type"])
    if rt == TypeId.BOOL8:
        ev = np.array([bool(v) for v in case["expect"]], dtype=bool)
    else:
        ev = np.array(case["expect"], dtype=storage_dtype(rt)) if case["expect"] else np.zeros(0, storage_dtype(rt))
    evv = None if case["expect_valid"] is None else np.array(case["expect_valid"], bool)
    key_tid = TypeId.DICTIONARY32 if case["key_dict"] else kt
    return {"num_groups": len(ek), "keys": [(int(key_tid), ek, ekv)], "results": [[(int(rt), ev, evv)]]}


def check_against_expected(got, case):
    want = expected(case)
    assert got["num_groups"] == want["num_groups"], f"{got['num_groups']} groups, expected {want['num_groups']}"
    go = T.sort_order(got["keys"])
    wo = T.sort_order(want["keys"])
    T.compare_keys(got["keys"], want["keys"], go, wo)
    # a QUANTILE result holds num_quantiles rows per group, group by group
    nq = len(case["extra"].get("quantiles", ())) if Kind(case["kind"]) == Kind.QUANTILE else 1
    go, wo = T.rows_of_groups(go, nq), T.rows_of_groups(wo, nq)
    T.compare_values(Kind(case["kind"]), got["results"][0][0], want["results"][0][0], go, wo, ctx=case["id"])


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_matches_reference_kat(case):
    keys, reqs = build(case)
    if case["keys_are_sorted"]:
        got = orc_sorted.groupby(keys, reqs, case["null_policy"])
    else:
        got = orc.groupby(keys, reqs, case["null_policy"])
    check_against_expected(got, case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_gpu_matches_reference_kat(case):
    keys, reqs = build(case)
    got = T.run_gpu(keys, reqs, case["null_policy"], keys_are_sorted=case["keys_are_sorted"])
    check_against_expected(got, case)


def test_oracle_mismatch_num_rows():
    """keys_tests.cpp:227-243: size mismatch is a logic_error."""
    c = KAT.mismatch_case()
    with pytest.raises(RuntimeError) as e:
        orc.groupby([HostCol(np.array(c["keys"], np.int32))], [(HostCol(np.array(c["values"], np.int32)),
                                                               [(Kind.COUNT_VALID, 0)])])
    assert "Size mismatch" in str(e.value)


def test_oracle_duplicate_aggregations_and_columns():
    """keys_tests.cpp:367-421: duplicate (column, agg) pairs are all answered."""
    k = HostCol(np.array(KAT.K10, np.int32))
    v = HostCol(np.array(KAT.V10, np.int32))
    r = orc.groupby([k], [(v, [(Kind.SUM, 0), (Kind.SUM, 0)]), (v, [(Kind.SUM, 0)])])
    a, b, c = r["results"][0][0][1], r["results"][0][1][1], r["results"][1][0][1]
    assert np.array_equal(a, b) and np.array_equal(a, c)
