"""Known answers of libcudf's stream-compaction and distinct-join gtests,
restated as data (libcudf 24.10):
  cpp/tests/stream_compaction/distinct_count_tests.cpp
  cpp/tests/stream_compaction/distinct_tests.cpp
  cpp/tests/join/distinct_join_tests.cpp
Columns are (values, valid or None).  In the distinct tests the payload
column holds each row's own index, so the expected rows are listed as row
indices.  The join tests' string key columns are written as integer codes
("s0" -> 0, "s1" -> 1, ...): equal strings get equal codes, so which rows
match is unchanged.
"""
from __future__ import annotations

import math

NaN = math.nan

# (id, columns, distinct_count EQUAL, distinct_count UNEQUAL)
DISTINCT_COUNT = [
    ("distinct_count_tests.cpp:265 TableWithNull",
     [([5, 4, 3, 5, 8, 1, 4, 5, 0, 9, -1], [1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0], "int32"),
      ([2, 2, 2, -1, 2, 1, 2, 0, 0, 9, -1], [1, 1, 1, 0, 1, 1, 1, 0, 0, 1, 0], "int32")], 8, 10),
    ("distinct_count_tests.cpp:279 TableWithSomeNull",
     [([1, 2, 3, 4, 5, 6], [1, 0, 1, 0, 1, 0], "int32"), ([1, 1, 1, 1, 1, 1], None, "int32")], 4, 6),
    ("distinct_count_tests.cpp:300 TableMixedTypes",
     [([5, 4, 3, 5, 8, 1, 4, 5, 0, 9, -1], [1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0], "int32"),
      ([2, 2, 2, -1, 2, 1, 2, 0, 0, 9, -1], [1, 1, 1, 0, 1, 1, 1, 0, 0, 1, 0], "float64"),
      ([2, 2, 2, 2 ** 32 - 1, 2, 1, 2, 0, 0, 9, 2 ** 32 - 1], [1, 1, 1, 0, 1, 1, 1, 1, 0, 1, 0], "uint32")], 9, 10),
]

# distinct_count_tests.cpp:67 TableNoNull: the answer is the number of distinct pairs
TABLE_NO_NULL = ([1, 3, 3, 3, 4, 31, 1, 8, 2, 0, 4, 1, 4, 10, 40, 31, 42, 0, 42, 8, 5, 4],
                 [3, 3, 3, 4, 31, 1, 8, 5, 0, 4, 1, 4, 10, 40, 31, 42, 0, 42, 8, 5, 4, 1])

# (id, key columns, nulls_equal, nans_equal, {keep: sorted expected rows})
# keep: 1 FIRST, 2 LAST, 3 NONE
DISTINCT = [
    ("distinct_tests.cpp:219 NoNullsTable",
     [([20, 20, 20, 20, 19, 21, 9], None, "int32"), ([19, 19, 19, 20, 20, 9, 21], None, "int32")], True, True,
     {1: [0, 3, 4, 5, 6], 2: [2, 3, 4, 5, 6], 3: [3, 4, 5, 6]}),
    ("distinct_tests.cpp:451 InputWithNullsEqual",
     [([20, 0, 0, 19, 21, 19, 22], [1, 0, 0, 1, 1, 1, 1], "int32")], True, True,
     {1: [0, 1, 3, 4, 6], 2: [0, 2, 4, 5, 6], 3: [0, 4, 6]}),
    ("distinct_tests.cpp:493 InputWithNullsUnequal",
     [([20, 0, 0, 19, 21, 19, 22, 20], [1, 0, 0, 1, 1, 1, 1, 1], "int32")], False, True,
     {1: [0, 1, 2, 3, 4, 6], 2: [1, 2, 4, 5, 6, 7], 3: [1, 2, 4, 6]}),
    ("distinct_tests.cpp:535 InputWithNaNsEqual",
     [([20., NaN, NaN, 19., 21., 19., 22.], None, "float32")], True, True,
     {1: [0, 1, 3, 4, 6], 2: [0, 2, 4, 5, 6], 3: [0, 4, 6]}),
    ("distinct_tests.cpp:577 InputWithNaNsUnequal",
     [([20., NaN, NaN, 19., 21., 19., 22., 20.], None, "float32")], False, False,
     {1: [0, 1, 2, 3, 4, 6], 2: [1, 2, 4, 5, 6, 7], 3: [1, 2, 4, 6]}),
]

# distinct_tests.cpp:179 NoNullsTableWithNaNs (KEEP_ANY): rows kept per nan_equality
ANY_WITH_NANS = ([([20, 20, 20, 15, 15, 15, 20, 19, 21, 9], None, "int32"),
                  ([19., 19., 19., NaN, NaN, NaN, 20., 20., 9., 21.], None, "float32")],
                 {False: 8, True: 6})

# (id, build key columns, probe key columns, nulls_equal, inner pairs sorted (build, probe)
#  or None, left: build row per probe row (None: no match) or None)
JOIN = [
    ("distinct_join_tests.cpp:106 InnerJoinNoNulls",
     [([1, 2, 3, 4, 5], None, "int32"), ([0, 0, 3, 4, 5], None, "int32"), ([9, 9, 9, 9, 9], None, "int32")],
     [([1, 2, 3, 4, 9], None, "int32"), ([0, 0, 0, 4, 4], None, "int32"), ([9, 9, 9, 0, 9], None, "int32")],
     True, [(0, 0), (1, 1)], None),
    ("distinct_join_tests.cpp:148 InnerJoinWithNulls",
     [([3, 1, 2, 0, 2], None, "int32"), ([1, 1, 0, 4, 0], [1, 1, 0, 1, 1], "int32"), ([1, 1, 2, 4, 1], None, "int32")],
     [([1, 2, 0, 2, 3], None, "int32"), ([1, 0, 1, 0, 1], None, "int32"), ([1, 1, 1, 1, 1], [0, 1, 1, 0, 1], "int32")],
     True, [(0, 4), (4, 1)], None),
    ("distinct_join_tests.cpp:370 LeftJoinNoNulls",
     [([2, 2, 0, 4, 3], None, "int32"), ([1, 0, 1, 2, 1], None, "int32")],
     [([3, 1, 2, 0, 3], None, "int32"), ([0, 1, 2, 4, 1], None, "int32")],
     True, None, [None, None, None, None, 4]),
    ("distinct_join_tests.cpp:406 LeftJoinWithNulls",
     [([2, 2, 0, 4, 3], None, "int32"), ([1, 0, 1, 2, 1], None, "int32")],
     [([3, 1, 2, 0, 2], None, "int32"), ([1, 1, 0, 4, 0], [1, 1, 0, 1, 1], "int32")],
     True, None, [4, None, None, None, 1]),
]


# STRING and STRUCT keys (column forms of tests/golden/struct_kats.py).
# distinct_tests.cpp:80-123 DistinctKeepFirstLastNone.StringKeyColumn: the
# kept rows of the key column {"all", "new", "new", "all", NULL, "the",
# "strings"} (nulls equal) per keep option.
STRING_KEY_COLUMN = ([("string", ["all", "new", "new", "all", "", "the", "strings"], [1, 1, 1, 1, 0, 1, 1])],
                     {1: [0, 1, 4, 5, 6], 2: [2, 3, 4, 5, 6], 3: [4, 5, 6]})
# distinct_tests.cpp:1204-1255 DistinctKeepAny.StructsOfStructs: s1{s2{a, b}, c}
# with s2 null at rows 2, 3, 7 and s1 null at rows 4, 5; KEEP_ANY keeps one row
# of each class: {0, 6}, {1}, {2}, {3, 7}, {4, 5}, {8} with nulls equal, and
# under nulls unequal every row holding a null stands alone.
_X = 0  # a placeholder under a null
STRUCTS_OF_STRUCTS = (
    [("struct", [("struct", [("fixed", "int32", [1, 1, _X, _X, _X, _X, 1, _X, 2], None),
                             ("fixed", "int32", [1, 2, _X, _X, _X, _X, 1, _X, 1], None)],
                  [1, 1, 0, 0, 1, 1, 1, 0, 1]),
                 ("fixed", "int32", [5, 4, 6, 4, _X, _X, 5, 4, 5], None)],
      [1, 1, 1, 1, 0, 0, 1, 1, 1])],
    {"equal": [[0, 6], [1], [2], [3, 7], [4, 5], [8]],
     "unequal": [[0, 6], [1], [2], [3], [7], [4], [5], [8]]})
