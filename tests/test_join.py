"""Hash joins on the CPU: the join oracle (oracle/join.py) against the
reference gtests' known answers (tests/golden/join_kats.py), and the C-ABI
argument checks of gbx_hash_join that need no GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cudf_b200 import _abi
from cudf_b200._abi import JoinKind, NullEquality, TypeId
from oracle import join as OJ
from tests.golden import join_kats as KAT
from tests.test_struct_keys import host_of

CASES = KAT.cases()


def keys_of(specs):
    return [host_of(s) for s in specs]


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_matches_join_kat(case):
    got = OJ.hash_join(keys_of(case["left"]), keys_of(case["right"]), case["nulls"], case["kind"])
    want = sorted(case["pairs"], key=lambda p: (-1 if p[0] is None else p[0], -1 if p[1] is None else p[1]))
    assert got == want


def test_oracle_nulls_unequal_in_struct_members():
    """Under UNEQUAL a null anywhere in the key matches nothing, a struct
    member included; under EQUAL the null members match."""
    m = [("fixed", TypeId.INT32, [1, 1], [1, 0])]
    left = [("struct", m, None)]
    right = [("struct", m, None)]
    assert OJ.hash_join(keys_of(left), keys_of(right), NullEquality.EQUAL) == [(0, 0), (1, 1)]
    assert OJ.hash_join(keys_of(left), keys_of(right), NullEquality.UNEQUAL) == [(0, 0)]


def test_hash_join_argument_checks():
    from cudf_b200 import _lib as L

    lib = L.lib()
    a = np.arange(4, dtype=np.int32)
    b = np.arange(4, dtype=np.int64)

    def table(arr, tid):
        v = _abi.gbx_column_view()
        v.type_id = int(tid)
        v.size = len(arr)
        v.data = arr.ctypes.data
        cols = (_abi.gbx_column_view * 1)(v)
        tv = _abi.gbx_table_view()
        tv.num_columns = 1
        tv.columns = C.cast(cols, C.POINTER(_abi.gbx_column_view))
        tv._keep = cols
        return tv

    l, r = table(a, TypeId.INT32), table(b, TypeId.INT64)
    li, ri = _abi.gbx_column(), _abi.gbx_column()
    # mismatched key types, bad kind, bad null equality: all before any CUDA call
    assert lib.gbx_hash_join(C.byref(l), C.byref(r), 0, 0, None, None, C.byref(li), C.byref(ri)) == \
        _abi.Status.ERR_LOGIC
    assert lib.gbx_hash_join(C.byref(l), C.byref(l), 0, 9, None, None, C.byref(li), C.byref(ri)) == \
        _abi.Status.ERR_LOGIC
    assert lib.gbx_hash_join(C.byref(l), C.byref(l), 5, 0, None, None, C.byref(li), C.byref(ri)) == \
        _abi.Status.ERR_LOGIC
    assert int(JoinKind.LEFT_ANTI) == 4
