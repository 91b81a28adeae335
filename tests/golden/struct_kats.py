"""Known answers of libcudf's STRUCT-key groupby gtests, restated as data.

Each case cites cpp/tests/groupby/structs_tests.cpp (libcudf 24.10).  The
literal inputs and expected outputs are the reference's; TYPED_TEST's member
type M1 (FixedWidthTypes there) is expanded over the fixed-width types this
library takes.  The harness (groupby_test_util.cpp:100-115, test_sum_agg)
groups with null_policy INCLUDE and compares results sorted by key.

A column is ("fixed", type_id, values, valid) / ("string", values, valid) /
("struct", [members], valid); valid None means no mask; a None element of a
values list stands where the reference writes a placeholder under a null.
"""
from __future__ import annotations

from cudf_b200._abi import TypeId as T

M1_TYPES = [T.INT8, T.INT16, T.INT32, T.INT64, T.UINT16, T.UINT64, T.FLOAT32, T.FLOAT64, T.BOOL8,
            T.TIMESTAMP_DAYS, T.DURATION_SECONDS]

V10 = list(range(10))
M0 = [1, 2, 3, 1, 2, 2, 1, 3, 3, 2]
M1 = [11, 22, 33, 11, 22, 22, 11, 33, 33, 22]
M2 = ["11", "22", "33", "11", "22", "22", "11", "33", "33", "22"]


def _nulls_at(n, idx):
    return [0 if i in idx else 1 for i in range(n)]


def _fx(t, vals, valid=None):
    return ("fixed", t, vals, valid)


def _st(vals, valid=None):
    return ("string", vals, valid)


def _sx(members, valid=None):
    return ("struct", members, valid)


def cases():
    out = []
    for t in M1_TYPES:
        # structs_tests.cpp:72-94 basic
        out.append(dict(
            id=f"structs_tests.cpp:72-94 basic[{t.name}]",
            keys=_sx([_fx(T.INT32, M0), _fx(t, M1), _st(M2)]), values=V10,
            expect_keys=_sx([_fx(T.INT32, [1, 2, 3]), _fx(t, [11, 22, 33]), _st(["11", "22", "33"])]),
            expect=[9, 19, 17]))
        # structs_tests.cpp:96-122 structs_with_nulls_in_members
        out.append(dict(
            id=f"structs_tests.cpp:96-122 structs_with_nulls_in_members[{t.name}]",
            keys=_sx([_fx(T.INT32, M0, _nulls_at(10, [1])), _fx(t, M1, _nulls_at(10, [7])), _st(M2)]), values=V10,
            expect_keys=_sx([_fx(T.INT32, [1, 2, 3, 3, None], _nulls_at(5, [4])),
                             _fx(t, [11, 22, 33, None, 22], _nulls_at(5, [3])),
                             _st(["11", "22", "33", "33", "22"])]),
            expect=[9, 18, 10, 7, 1]))
        # structs_tests.cpp:124-148 structs_with_null_rows
        out.append(dict(
            id=f"structs_tests.cpp:124-148 structs_with_null_rows[{t.name}]",
            keys=_sx([_fx(T.INT32, M0), _fx(t, M1), _st(M2)], _nulls_at(10, [0, 3])), values=V10,
            expect_keys=_sx([_fx(T.INT32, [1, 2, 3, None], _nulls_at(4, [3])),
                             _fx(t, [11, 22, 33, None], _nulls_at(4, [3])),
                             _st(["11", "22", "33", None], _nulls_at(4, [3]))], _nulls_at(4, [3])),
            expect=[6, 19, 17, 3]))
        # structs_tests.cpp:150-177 structs_with_nulls_in_rows_and_members
        out.append(dict(
            id=f"structs_tests.cpp:150-177 structs_with_nulls_in_rows_and_members[{t.name}]",
            keys=_sx([_fx(T.INT32, M0, _nulls_at(10, [1])), _fx(t, M1, _nulls_at(10, [7])), _st(M2)],
                     _nulls_at(10, [4])), values=V10,
            expect_keys=_sx([_fx(T.INT32, [1, 2, 3, 3, None, None], _nulls_at(6, [4, 5])),
                             _fx(t, [11, 22, 33, None, 22, None], _nulls_at(6, [3, 5])),
                             _st(["11", "22", "33", "33", "22", None], _nulls_at(6, [5]))], _nulls_at(6, [5])),
            expect=[9, 14, 10, 7, 1, 4]))
        # structs_tests.cpp:179-211 null_members_differ_from_null_structs
        out.append(dict(
            id=f"structs_tests.cpp:179-211 null_members_differ_from_null_structs[{t.name}]",
            keys=_sx([_fx(T.INT32, M0, _nulls_at(10, [1])), _fx(t, M1, _nulls_at(10, [1])),
                      _st(M2, _nulls_at(10, [1]))], _nulls_at(10, [4])), values=V10,
            expect_keys=_sx([_fx(T.INT32, [1, 2, 3, None, None], _nulls_at(5, [3, 4])),
                             _fx(t, [11, 22, 33, None, None], _nulls_at(5, [3, 4])),
                             _st(["11", "22", "33", None, None], _nulls_at(5, [3, 4]))], _nulls_at(5, [4])),
            expect=[9, 14, 17, 1, 4]))
        # structs_tests.cpp:213-247 structs_of_structs
        inner = _sx([_fx(T.INT32, M0, _nulls_at(10, [1])), _fx(t, M1, _nulls_at(10, [1])),
                     _st(M2, _nulls_at(10, [1]))], _nulls_at(10, [4]))
        out.append(dict(
            id=f"structs_tests.cpp:213-247 structs_of_structs[{t.name}]",
            keys=_sx([inner, _fx(t, [8, 9, 6, 8, 0, 7, 8, 6, 6, 7])]), values=V10,
            expect_keys=_sx([_sx([_fx(T.INT32, [1, 2, 3, None, None], _nulls_at(5, [3, 4])),
                                  _fx(t, [11, 22, 33, None, None], _nulls_at(5, [3, 4])),
                                  _st(["11", "22", "33", None, None], _nulls_at(5, [3, 4]))], _nulls_at(5, [4])),
                             _fx(t, [8, 7, 6, 9, 0])]),
            expect=[9, 14, 17, 1, 4]))
        # structs_tests.cpp:249-271 empty_input
        out.append(dict(
            id=f"structs_tests.cpp:249-271 empty_input[{t.name}]",
            keys=_sx([_fx(T.INT32, []), _fx(t, []), _st([])]), values=[],
            expect_keys=_sx([_fx(T.INT32, []), _fx(t, []), _st([])]), expect=[]))
        # structs_tests.cpp:273-295 all_null_input
        out.append(dict(
            id=f"structs_tests.cpp:273-295 all_null_input[{t.name}]",
            keys=_sx([_fx(T.INT32, M0), _fx(t, M1), _st(M2)], [0] * 10), values=V10,
            expect_keys=_sx([_fx(T.INT32, [None], [0]), _fx(t, [None], [0]), _st([None], [0])], [0]),
            expect=[45]))
    return out
