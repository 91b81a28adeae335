"""Known answers of libcudf's join gtests, restated as data.

Each case cites cpp/tests/join/join_tests.cpp or semi_anti_join_tests.cpp
(libcudf 24.10).  The reference tests gather both tables with the returned
maps and compare the joined rows sorted; here the expected result is the set
of (left row, right row) pairs those gold tables are made of (None where the
reference's gather gives nulls: cudf::JoinNoneValue).  Key columns use the
struct_kats column forms: ("fixed", type_id, values, valid),
("string", values, valid), ("struct", [members], valid).
"""
from __future__ import annotations

from cudf_b200._abi import JoinKind as J, NullEquality as E, TypeId as T

# the tables of FullJoin* / LeftJoinNoNulls (join_tests.cpp:227-470), key
# columns 0 and 1
L_A = [("fixed", T.INT32, [3, 1, 2, 0, 3], None), ("string", ["s0", "s1", "s2", "s4", "s1"], None)]
R_A = [("fixed", T.INT32, [2, 2, 0, 4, 3], None), ("string", ["s1", "s0", "s1", "s2", "s1"], None)]
R_A_NULL = [("fixed", T.INT32, [2, 2, 0, 4, 3], [1, 1, 1, 0, 1]), ("string", ["s1", "s0", "s1", "s2", "s1"], None)]
# InnerJoin* (join_tests.cpp:701-960)
L_B = [("fixed", T.INT32, [3, 1, 2, 0, 2], None), ("string", ["s1", "s1", "s0", "s4", "s0"], None)]
R_B = [("fixed", T.INT32, [2, 2, 0, 4, 3], None), ("string", ["s1", "s0", "s1", "s2", "s1"], None)]
L_ON_NULLS = [("fixed", T.INT32, [3, 1, 2, 0, 2], None),
              ("string", ["s1", "s1", "s8", "s4", "s0"], [1, 1, 0, 1, 1])]
R_ON_NULLS = [("fixed", T.INT32, [2, 2, 0, 4, 3], None),
              ("string", ["s1", "s0", "s1", "s2", "s1"], [1, 0, 1, 1, 1])]
# LeftJoinWithNulls (join_tests.cpp:470-514)
L_C = [("fixed", T.INT32, [3, 1, 2, 0, 2], None), ("string", ["s1", "s1", "", "s4", "s0"], [1, 1, 0, 1, 1])]
# InnerJoinWithStructsAndNulls (join_tests.cpp:791-877), key columns 0, 1, 3
L_S = [("fixed", T.INT32, [3, 1, 2, 0, 2], None), ("string", ["s1", "s1", "s0", "s4", "s0"], [1, 1, 0, 1, 1]),
       ("struct", [("string", ["Samuel Vimes", "Carrot Ironfoundersson", "Detritus", "Samuel Vimes",
                               "Angua von Überwald"], None),
                   ("fixed", T.INT32, [48, 27, 351, 31, 25], None),
                   ("fixed", T.BOOL8, [1, 1, 0, 0, 0], [1, 1, 0, 1, 0])], None)]
R_S = [("fixed", T.INT32, [2, 2, 0, 4, 3], None), ("string", ["s1", "s0", "s1", "s2", "s1"], None),
       ("struct", [("string", ["Carrot Ironfoundersson", "Angua von Überwald", "Detritus", "Carrot Ironfoundersson",
                               "Samuel Vimes"], None),
                   ("fixed", T.INT32, [351, 25, 27, 31, 48], None),
                   ("fixed", T.BOOL8, [1, 0, 0, 0, 1], [1, 0, 0, 1, 1])], None)]
EQ2 = [("fixed", T.INT32, [0, 0], None), ("string", ["s0", "s0"], None)]
# the Empty* tests (join_tests.cpp:962-1225)
E_2 = [("fixed", T.INT32, [], None), ("fixed", T.INT32, [], None)]
T_2 = [("fixed", T.INT32, [2, 2, 0, 4, 3], None), ("fixed", T.INT32, [1, 0, 1, 2, 1], [1, 0, 1, 1, 1])]
N = None


def cases():
    return [
        dict(id="join_tests.cpp:227-278 FullJoinNoNulls", left=L_A, right=R_A, kind=J.FULL, nulls=E.EQUAL,
             pairs=[(0, N), (1, N), (2, N), (3, N), (4, 4), (N, 0), (N, 1), (N, 2), (N, 3)]),
        dict(id="join_tests.cpp:280-331 FullJoinWithNulls", left=L_A, right=R_A_NULL, kind=J.FULL, nulls=E.EQUAL,
             pairs=[(0, N), (1, N), (2, N), (3, N), (4, 4), (N, 0), (N, 1), (N, 2), (N, 3)]),
        dict(id="join_tests.cpp:425-468 LeftJoinNoNulls", left=L_A, right=R_A, kind=J.LEFT, nulls=E.EQUAL,
             pairs=[(0, N), (1, N), (2, N), (3, N), (4, 4)]),
        dict(id="join_tests.cpp:470-514 LeftJoinWithNulls", left=L_C, right=R_B, kind=J.LEFT, nulls=E.EQUAL,
             pairs=[(0, 4), (1, N), (2, N), (3, N), (4, 1)]),
        dict(id="join_tests.cpp:701-744 InnerJoinNoNulls", left=L_B, right=R_B, kind=J.INNER, nulls=E.EQUAL,
             pairs=[(0, 4), (2, 1), (4, 1)]),
        dict(id="join_tests.cpp:791-877 InnerJoinWithStructsAndNulls", left=L_S, right=R_S, kind=J.INNER,
             nulls=E.EQUAL, pairs=[(0, 4), (4, 1)]),
        dict(id="join_tests.cpp:879-960 InnerJoinOnNulls (nulls equal)", left=L_ON_NULLS, right=R_ON_NULLS,
             kind=J.INNER, nulls=E.EQUAL, pairs=[(0, 4), (2, 1)]),
        dict(id="join_tests.cpp:879-960 InnerJoinOnNulls (nulls unequal)", left=L_ON_NULLS, right=R_ON_NULLS,
             kind=J.INNER, nulls=E.UNEQUAL, pairs=[(0, 4)]),
        dict(id="join_tests.cpp:1227-1260 EqualValuesInnerJoin", left=EQ2, right=EQ2, kind=J.INNER, nulls=E.EQUAL,
             pairs=[(0, 0), (0, 1), (1, 0), (1, 1)]),
        dict(id="join_tests.cpp:1262-1294 EqualValuesLeftJoin", left=EQ2, right=EQ2, kind=J.LEFT, nulls=E.EQUAL,
             pairs=[(0, 0), (0, 1), (1, 0), (1, 1)]),
        dict(id="join_tests.cpp:1296-1328 EqualValuesFullJoin", left=EQ2, right=EQ2, kind=J.FULL, nulls=E.EQUAL,
             pairs=[(0, 0), (0, 1), (1, 0), (1, 1)]),
        dict(id="semi_anti_join_tests.cpp:96-114 TestSimple (semi)", left=[("fixed", T.INT32, [0, 1, 2], None)],
             right=[("fixed", T.INT32, [0, 1, 3], None)], kind=J.LEFT_SEMI, nulls=E.EQUAL, pairs=[(0, N), (1, N)]),
        dict(id="semi_anti_join_tests.cpp:96-114 TestSimple inputs, anti join (the semi result's complement)", left=[("fixed", T.INT32, [0, 1, 2], None)],
             right=[("fixed", T.INT32, [0, 1, 3], None)], kind=J.LEFT_ANTI, nulls=E.EQUAL, pairs=[(2, N)]),
        dict(id="join_tests.cpp:962-981 EmptyLeftTableInnerJoin", left=E_2, right=T_2, kind=J.INNER, nulls=E.EQUAL,
             pairs=[]),
        dict(id="join_tests.cpp:1004-1042 EmptyLeftTableFullJoin", left=E_2, right=T_2, kind=J.FULL, nulls=E.EQUAL,
             pairs=[(N, 0), (N, 1), (N, 2), (N, 3), (N, 4)]),
        dict(id="join_tests.cpp:1083-1120 EmptyRightTableLeftJoin", left=T_2, right=E_2, kind=J.LEFT, nulls=E.EQUAL,
             pairs=[(0, N), (1, N), (2, N), (3, N), (4, N)]),
    ]
