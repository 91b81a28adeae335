"""Known-answer vectors of libcudf's groupby gtests, restated as data.

Each case cites the reference test it comes from (cpp/tests/groupby/*.cpp,
libcudf 24.10).  The literal inputs and expected outputs are the reference's;
the typed-test expansion mirrors its TYPED_TEST_SUITE type lists for the
types this library supports.  Comparison follows the reference harness
(cpp/tests/groupby/groupby_test_util.cpp:89-96): results are sorted by key
before comparing, and floating values are compared "equivalent"
(cpp/tests/utilities/column_utilities.cu:406-425, 4 ulp) -- here with a
relative tolerance stated in the test.
"""
from __future__ import annotations

import math

from cudf_b200._abi import Kind, NullPolicy, TypeId as T

INTS = [T.INT8, T.INT16, T.INT32, T.INT64]
FLOATS = [T.FLOAT32, T.FLOAT64]
DURATIONS = [T.DURATION_DAYS, T.DURATION_SECONDS, T.DURATION_MILLISECONDS]
TIMESTAMPS = [T.TIMESTAMP_DAYS, T.TIMESTAMP_SECONDS]
UINTS = [T.UINT8, T.UINT16, T.UINT32, T.UINT64]

# Common literal inputs of the gtests.
K10 = [1, 2, 3, 1, 2, 2, 1, 3, 3, 2]
V10 = list(range(10))
K11 = [1, 2, 3, 1, 2, 2, 1, 3, 3, 2, 4]
K11_VALID = [1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 1]
V11 = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4]
V11_VALID_A = [0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0]  # sum/count/min/mean tests
V11_VALID_MAX = [1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 0]  # max_tests.cpp:117-118
V11_VAR = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 3]
V11_VALID_VAR = [0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1]


def sum_type(v):
    if v in INTS or v in UINTS or v == T.BOOL8:
        return T.INT64
    return v


def _case(cid, ktype, keys, vtype, vals, kind, expect_keys, expect, *, kvalid=None, vvalid=None, evalid=None,
          ekvalid=None, ddof=0, null_policy=NullPolicy.EXCLUDE, rtype=None, vdict=False, kdict=False,
          float_expect=False, extra=None, offset=0, size=None, keys_are_sorted=False):
    """`null_policy` is the groupby's; `extra` holds an aggregation's own
    null_policy / interpolation / quantiles; `offset` and `size` slice both
    columns (a column view of rows offset .. offset + size);
    `keys_are_sorted` is the groupby's sorted::YES."""
    return dict(
        id=cid, key_type=ktype, keys=keys, key_valid=kvalid, key_dict=kdict,
        value_type=vtype, values=vals, value_valid=vvalid, value_dict=vdict,
        kind=kind, ddof=ddof, null_policy=null_policy,
        expect_keys=expect_keys, expect_key_valid=ekvalid,
        expect=expect, expect_valid=evalid, result_type=rtype, float_expect=float_expect,
        extra=extra or {}, offset=offset, size=size, keys_are_sorted=keys_are_sorted,
    )


def cases():
    out = []
    K = T.INT32
    # ---- sum_tests.cpp (supported_types: int8..int64, float, double, durations)
    for v in INTS + FLOATS + DURATIONS:
        r = sum_type(v)
        out += [
            _case(f"sum_tests.cpp:38-54 basic[{v.name}]", K, K10, v, V10, Kind.SUM, [1, 2, 3], [9, 19, 17], rtype=r),
            _case(f"sum_tests.cpp:56-72 empty_cols[{v.name}]", K, [], v, [], Kind.SUM, [], [], rtype=r),
            _case(f"sum_tests.cpp:74-90 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.SUM, [], [],
                  kvalid=[0, 0, 0], rtype=r),
            _case(f"sum_tests.cpp:92-108 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.SUM, [1], [0],
                  vvalid=[0, 0, 0], evalid=[0], rtype=r),
            _case(f"sum_tests.cpp:110-132 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.SUM, [1, 2, 3, 4],
                  [9, 14, 10, 0], kvalid=K11_VALID, vvalid=V11_VALID_A, evalid=[1, 1, 1, 0], rtype=r),
        ]
        if v not in DURATIONS:
            out.append(_case(f"sum_tests.cpp:134-152 dictionary[{v.name}]", K, K10, v, V10, Kind.SUM, [1, 2, 3],
                             [9, 19, 17], rtype=r, vdict=True))
    out.append(_case("sum_tests.cpp:155-172 overflow_integer", T.INT32, [0, 0], T.INT32, [-2147483648, -2147483648],
                     Kind.SUM, [0], [-4294967296], rtype=T.INT64))

    # ---- count_tests.cpp (AllTypes; fixed-width members)
    for v in INTS + UINTS + FLOATS + [T.BOOL8] + TIMESTAMPS + DURATIONS + [T.DECIMAL32, T.DECIMAL64]:
        out += [
            _case(f"count_tests.cpp:32-52 basic[{v.name}]", K, K10, v, V10, Kind.COUNT_VALID, [1, 2, 3], [3, 4, 3],
                  rtype=T.INT32),
            _case(f"count_tests.cpp:32-52 basic_include[{v.name}]", K, K10, v, V10, Kind.COUNT_ALL, [1, 2, 3],
                  [3, 4, 3], rtype=T.INT32),
            _case(f"count_tests.cpp:54-69 empty_cols[{v.name}]", K, [], v, [], Kind.COUNT_VALID, [], [],
                  rtype=T.INT32),
            _case(f"count_tests.cpp:71-90 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.COUNT_VALID,
                  [], [], kvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"count_tests.cpp:71-90 zero_valid_keys_include[{v.name}]", K, [1, 2, 3], v, [3, 4, 5],
                  Kind.COUNT_ALL, [], [], kvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"count_tests.cpp:92-114 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.COUNT_VALID,
                  [1], [0], vvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"count_tests.cpp:92-114 zero_valid_values_include[{v.name}]", K, [1, 1, 1], v, [3, 4, 5],
                  Kind.COUNT_ALL, [1], [3], vvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"count_tests.cpp:116-145 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.COUNT_VALID,
                  [1, 2, 3, 4], [2, 3, 2, 0], kvalid=K11_VALID, vvalid=V11_VALID_A, rtype=T.INT32),
            _case(f"count_tests.cpp:116-145 null_keys_and_values_include[{v.name}]", K, K11, v, V11, Kind.COUNT_ALL,
                  [1, 2, 3, 4], [3, 4, 2, 1], kvalid=K11_VALID, vvalid=V11_VALID_A, rtype=T.INT32),
        ]

    # ---- min_tests.cpp / max_tests.cpp (FixedWidthTypesWithoutFixedPoint)
    for v in INTS + UINTS + FLOATS + [T.BOOL8] + TIMESTAMPS + DURATIONS:
        out += [
            _case(f"min_tests.cpp:37-52 basic[{v.name}]", K, K10, v, V10, Kind.MIN, [1, 2, 3], [0, 1, 2], rtype=v),
            _case(f"min_tests.cpp:54-69 empty_cols[{v.name}]", K, [], v, [], Kind.MIN, [], [], rtype=v),
            _case(f"min_tests.cpp:71-88 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.MIN, [], [],
                  kvalid=[0, 0, 0], rtype=v),
            _case(f"min_tests.cpp:90-107 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.MIN, [1], [0],
                  vvalid=[0, 0, 0], evalid=[0], rtype=v),
            _case(f"min_tests.cpp:109-132 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.MIN, [1, 2, 3, 4],
                  [3, 1, 2, 0], kvalid=K11_VALID, vvalid=V11_VALID_A, evalid=[1, 1, 1, 0], rtype=v),
            _case(f"max_tests.cpp:37-53 basic[{v.name}]", K, K10, v, V10, Kind.MAX, [1, 2, 3], [6, 9, 8], rtype=v),
            _case(f"max_tests.cpp:55-71 empty_cols[{v.name}]", K, [], v, [], Kind.MAX, [], [], rtype=v),
            _case(f"max_tests.cpp:73-89 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.MAX, [], [],
                  kvalid=[0, 0, 0], rtype=v),
            _case(f"max_tests.cpp:91-107 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.MAX, [1], [0],
                  vvalid=[0, 0, 0], evalid=[0], rtype=v),
            _case(f"max_tests.cpp:109-130 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.MAX, [1, 2, 3, 4],
                  [3, 5, 8, 0], kvalid=K11_VALID, vvalid=V11_VALID_MAX, evalid=[1, 1, 1, 0], rtype=v),
        ]
    # ---- argmin_tests.cpp / argmax_tests.cpp (FixedWidthTypes; the gtests skip
    # bool, and fixed-point needs a scale the wrapper here does not carry)
    vdesc = [9, 8, 7, 6, 5, 4, 3, 2, 1, 0]
    vdesc11 = vdesc + [4]
    for v in INTS + UINTS + FLOATS + TIMESTAMPS + DURATIONS:
        out += [
            _case(f"argmin_tests.cpp:34-52 basic[{v.name}]", K, K10, v, vdesc, Kind.ARGMIN, [1, 2, 3], [6, 9, 8],
                  rtype=T.INT32),
            _case(f"argmin_tests.cpp:54-72 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.ARGMIN, [], [],
                  kvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"argmin_tests.cpp:74-92 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.ARGMIN, [1],
                  [0], vvalid=[0, 0, 0], evalid=[0], rtype=T.INT32),
            _case(f"argmin_tests.cpp:94-118 null_keys_and_values[{v.name}]", K, K11, v, vdesc11, Kind.ARGMIN,
                  [1, 2, 3, 4], [3, 9, 8, 0], kvalid=K11_VALID, vvalid=[1, 1, 1, 1, 1, 0, 0, 1, 1, 1, 0],
                  evalid=[1, 1, 1, 0], rtype=T.INT32),
            _case(f"argmax_tests.cpp:33-51 basic[{v.name}]", K, K10, v, vdesc, Kind.ARGMAX, [1, 2, 3], [0, 1, 2],
                  rtype=T.INT32),
            _case(f"argmax_tests.cpp:53-71 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.ARGMAX, [], [],
                  kvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"argmax_tests.cpp:73-91 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.ARGMAX, [1],
                  [0], vvalid=[0, 0, 0], evalid=[0], rtype=T.INT32),
            _case(f"argmax_tests.cpp:93-117 null_keys_and_values[{v.name}]", K, K11, v, vdesc11, Kind.ARGMAX,
                  [1, 2, 3, 4], [3, 4, 7, 0], kvalid=[1, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1],
                  vvalid=[0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 0], evalid=[1, 1, 1, 0], rtype=T.INT32),
        ]
    dvals = [0xABC, 0xBBB, 0xF1, 0xAAA, 0xFFF, 0xBAA, 0xAAA, 0x01, 0xF1, 0xEEE]
    out += [
        _case("min_tests.cpp:232-255 dictionary fixed_width", K, K10, T.INT64, dvals, Kind.MIN, [1, 2, 3],
              [0xAAA, 0xBAA, 0x01], rtype=T.INT64, vdict=True),
        _case("max_tests.cpp:235-258 dictionary fixed_width", K, K10, T.INT64, dvals, Kind.MAX, [1, 2, 3],
              [0xABC, 0xFFF, 0xF1], rtype=T.INT64, vdict=True),
    ]
    for v in FLOATS:
        # min_tests.cpp:529-552 / max_tests.cpp:533-556: must not hang; one group.
        # The value is NaN under this library's stated NaN order.
        out += [
            _case(f"min_tests.cpp:529-552 values_with_nan[{v.name}]", K, [1, 1], v, [math.nan, math.nan], Kind.MIN,
                  [1], [math.nan], rtype=v, float_expect=True),
            _case(f"max_tests.cpp:533-556 values_with_nan[{v.name}]", K, [1, 1], v, [math.nan, math.nan], Kind.MAX,
                  [1], [math.nan], rtype=v, float_expect=True),
        ]

    # ---- mean_tests.cpp (int8..int64, float, double, durations)
    for v in INTS + FLOATS + DURATIONS:
        dur = v in DURATIONS
        r = v if dur else T.FLOAT64
        basic = [3, 4, 5] if dur else [3.0, 19.0 / 4, 17.0 / 3]
        nk = [4, 4, 5, 0] if dur else [4.5, 14.0 / 3, 5.0, 0.0]
        out += [
            _case(f"mean_tests.cpp:48-64 basic[{v.name}]", K, K10, v, V10, Kind.MEAN, [1, 2, 3], basic, rtype=r,
                  float_expect=not dur),
            _case(f"mean_tests.cpp:66-80 empty_cols[{v.name}]", K, [], v, [], Kind.MEAN, [], [], rtype=r),
            _case(f"mean_tests.cpp:82-96 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], Kind.MEAN, [], [],
                  kvalid=[0, 0, 0], rtype=r),
            _case(f"mean_tests.cpp:98-111 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], Kind.MEAN, [1],
                  [0], vvalid=[0, 0, 0], evalid=[0], rtype=r),
            _case(f"mean_tests.cpp:113-139 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.MEAN, [1, 2, 3, 4],
                  nk, kvalid=K11_VALID, vvalid=V11_VALID_A, evalid=[1, 1, 1, 0], rtype=r, float_expect=not dur),
        ]
    out.append(_case("mean_tests.cpp:141-159 dictionary[INT16]", K, K10, T.INT16, V10, Kind.MEAN, [1, 2, 3],
                     [9.0 / 3, 19.0 / 4, 17.0 / 3], rtype=T.FLOAT64, vdict=True, float_expect=True))
    for dec in (T.DECIMAL32, T.DECIMAL64):
        for scale in (2, 1, 0, -1, -2):
            c = _case(f"mean_tests.cpp:186-207 GroupByHashMeanDecimalAsValue[{dec.name},scale={scale}]", K, K10, dec,
                      V10, Kind.MEAN, [1, 2, 3], [3, 4, 5], rtype=dec)
            c["value_scale"] = scale
            out.append(c)
            c = _case(f"sum_tests.cpp:208-232 GroupByHashSumDecimalAsValue[{dec.name},scale={scale}]", K, K10, dec,
                      V10, Kind.SUM, [1, 2, 3], [9, 19, 17], rtype=dec)
            c["value_scale"] = scale
            out.append(c)

    # ---- var_tests.cpp / std_tests.cpp (int8..int64, float, double)
    for v in INTS + FLOATS:
        for kind, f, tag in ((Kind.VARIANCE, lambda x: x, "var"), (Kind.STD, math.sqrt, "std")):
            out += [
                _case(f"{tag}_tests.cpp:35-53 basic[{v.name}]", K, K10, v, V10, kind, [1, 2, 3],
                      [f(9.0), f(131.0 / 12), f(31.0 / 3)], evalid=[1, 1, 1], rtype=T.FLOAT64, ddof=1,
                      float_expect=True),
                _case(f"{tag}_tests.cpp:55-69 empty_cols[{v.name}]", K, [], v, [], kind, [], [], rtype=T.FLOAT64,
                      ddof=1),
                _case(f"{tag}_tests.cpp:71-85 zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], kind, [], [],
                      kvalid=[0, 0, 0], rtype=T.FLOAT64, ddof=1),
                _case(f"{tag}_tests.cpp:87-101 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], kind, [1],
                      [0.0], vvalid=[0, 0, 0], evalid=[0], rtype=T.FLOAT64, ddof=1),
                _case(f"{tag}_tests.cpp:103-124 null_keys_and_values[{v.name}]", K, K11, v, V11_VAR, kind,
                      [1, 2, 3, 4], [f(4.5), f(49.0 / 3), f(18.0), 0.0], kvalid=K11_VALID, vvalid=V11_VALID_VAR,
                      evalid=[1, 1, 1, 0], rtype=T.FLOAT64, ddof=1, float_expect=True),
                _case(f"{tag}_tests.cpp:126-148 ddof_non_default[{v.name}]", K, K11, v, V11_VAR, kind,
                      [1, 2, 3, 4], [0.0, f(98.0 / 3), 0.0, 0.0], kvalid=K11_VALID, vvalid=V11_VALID_VAR,
                      evalid=[0, 1, 0, 0], rtype=T.FLOAT64, ddof=2, float_expect=True),
                _case(f"{tag}_tests.cpp:150-173 dictionary[{v.name}]", K, K10, v, V10, kind, [1, 2, 3],
                      [f(9.0), f(131.0 / 12), f(31.0 / 3)], evalid=[1, 1, 1], rtype=T.FLOAT64, ddof=1, vdict=True,
                      float_expect=True),
            ]
    out.append(_case("var_tests.cpp:175-200 sort_vs_hash", K, [50, 30, 90, 80], T.FLOAT64, [380.0, 370.0, 24.0, 26.0],
                     Kind.VARIANCE, [30, 50, 80, 90], [0.0, 0.0, 0.0, 0.0], evalid=[0, 0, 0, 0], rtype=T.FLOAT64,
                     ddof=1, float_expect=True))

    # ---- keys_tests.cpp (K: int8..int64, float, double, decimal32, decimal64; V = int32)
    for kt in INTS + FLOATS + [T.DECIMAL32, T.DECIMAL64]:
        V = T.INT32
        out += [
            _case(f"keys_tests.cpp:37-53 basic[{kt.name}]", kt, K10, V, V10, Kind.COUNT_VALID, [1, 2, 3], [3, 4, 3],
                  rtype=T.INT32),
            _case(f"keys_tests.cpp:55-71 zero_valid_keys[{kt.name}]", kt, [1, 2, 3], V, [3, 4, 5], Kind.COUNT_VALID,
                  [], [], kvalid=[0, 0, 0], rtype=T.INT32),
            _case(f"keys_tests.cpp:73-92 some_null_keys[{kt.name}]", kt, K11, V, V11, Kind.COUNT_VALID, [1, 2, 3, 4],
                  [3, 4, 2, 1], kvalid=K11_VALID, rtype=T.INT32),
            _case(f"keys_tests.cpp:94-120 include_null_keys[{kt.name}]", kt, K11, V, V11, Kind.SUM, [1, 2, 3, 4, 3],
                  [9, 19, 10, 4, 7], kvalid=K11_VALID, ekvalid=[1, 1, 1, 1, 0], null_policy=NullPolicy.INCLUDE,
                  rtype=T.INT64),
            # sorted::YES: groups are the runs of equal adjacent rows (under
            # INCLUDE a null run between two runs is a group of its own)
            _case(f"keys_tests.cpp:122-145 pre_sorted_keys[{kt.name}]", kt, [1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4], V,
                  V11, Kind.SUM, [1, 2, 3, 4], [3, 18, 24, 4], rtype=T.INT64, keys_are_sorted=True),
            _case(f"keys_tests.cpp:147-171 pre_sorted_keys_descending[{kt.name}]", kt,
                  [4, 3, 3, 3, 2, 2, 2, 2, 1, 1, 1], V, V11, Kind.SUM, [4, 3, 2, 1], [0, 6, 22, 21], rtype=T.INT64,
                  keys_are_sorted=True),
            _case(f"keys_tests.cpp:173-197 pre_sorted_keys_nullable[{kt.name}]", kt,
                  [1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4], V, V11, Kind.SUM, [1, 2, 3, 4], [3, 15, 17, 4],
                  kvalid=[1, 1, 1, 0, 1, 1, 1, 0, 1, 1, 1], rtype=T.INT64, keys_are_sorted=True),
            _case(f"keys_tests.cpp:199-225 pre_sorted_keys_nulls_before_include_nulls[{kt.name}]", kt,
                  [1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4], V, V11, Kind.SUM, [1, 2, 2, 3, 3, 4],
                  [3, 7, 11, 7, 17, 4], kvalid=[1, 1, 1, 0, 0, 1, 1, 0, 1, 1, 1], ekvalid=[1, 0, 1, 0, 1, 1],
                  null_policy=NullPolicy.INCLUDE, rtype=T.INT64, keys_are_sorted=True),
        ]
    # keys_tests.cpp:338-365: dictionary keys {"aaa","año","₹1"}; indices into the
    # sorted dictionary keys, values summed per dictionary entry.
    out.append(_case("keys_tests.cpp:338-365 dictionary_keys basic", T.INT32, [0, 1, 2, 0, 1, 1, 0, 2, 2, 1], T.INT32,
                     V10, Kind.SUM, [0, 1, 2], [9, 19, 17], rtype=T.INT64, kdict=True))
    out += sort_path_cases()
    # keys_tests.cpp:318-333 groupby_string_keys_test basic: STRING keys
    out.append(_case("keys_tests.cpp:318-333 string_keys basic", T.STRING,
                     ["aaa", "año", "₹1", "aaa", "año", "año", "aaa", "₹1", "₹1", "año"], T.INT32, V10, Kind.SUM,
                     ["aaa", "año", "₹1"], [9, 19, 17], rtype=T.INT64))
    return out


# The kinds libcudf computes on its sort path.  Groups come out in hash order
# here, so, like the cases above, they are compared sorted by key.
ALL_TYPES = INTS + UINTS + FLOATS + [T.BOOL8] + DURATIONS + TIMESTAMPS + [T.DECIMAL32, T.DECIMAL64]
K14 = [1, 2, 3, 3, 1, 2, 2, 1, 3, 3, 2, 4, 4, 2]
K14_VALID = [1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1]
V14 = [0, 1, 2, 2, 3, 4, 5, 6, 7, 8, 9, 4, 4, 2]
V14_VALID_NUNIQUE = [0, 1, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0, 0, 0]   # nunique_tests.cpp:154-155
V14_VALID_NTH = [0, 1, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1, 0, 0]       # nth_element_tests.cpp:215-216


def _q(quantiles, interp=0):
    return {"quantiles": list(quantiles), "interpolation": interp}


def sort_path_cases():
    out = []
    K = T.INT32
    F = T.FLOAT64
    # ---- median_tests.cpp and quantile_tests.cpp (int8..int64, float, double)
    for v in INTS + FLOATS:
        for tag, kind, ex, lines in (("median", Kind.MEDIAN, None, (35, 55, 71, 87, 103, 124)),
                                     ("quantile", Kind.QUANTILE, _q([0.5]), (36, 56, 72, 88, 104, 194))):
            b, e, zk, zv, nk, d = lines
            out += [
                _case(f"{tag}_tests.cpp:{b} basic[{v.name}]", K, K10, v, V10, kind, [1, 2, 3], [3.0, 4.5, 7.0],
                      rtype=F, extra=ex),
                _case(f"{tag}_tests.cpp:{e} empty_cols[{v.name}]", K, [], v, [], kind, [], [], rtype=F, extra=ex),
                _case(f"{tag}_tests.cpp:{zk} zero_valid_keys[{v.name}]", K, [1, 2, 3], v, [3, 4, 5], kind, [], [],
                      kvalid=[0, 0, 0], rtype=F, extra=ex),
                _case(f"{tag}_tests.cpp:{zv} zero_valid_values[{v.name}]", K, [1, 1, 1], v, [3, 4, 5], kind, [1],
                      [0.0], vvalid=[0, 0, 0], evalid=[0], rtype=F, extra=ex),
                _case(f"{tag}_tests.cpp:{nk} null_keys_and_values[{v.name}]", K, K11, v, V11, kind, [1, 2, 3, 4],
                      [4.5, 4.0, 5.0, 0.0], kvalid=K11_VALID, vvalid=V11_VALID_A, evalid=[1, 1, 1, 0], rtype=F,
                      extra=ex),
                _case(f"{tag}_tests.cpp:{d} dictionary[{v.name}]", K, K10, v, V10, kind, [1, 2, 3], [3.0, 4.5, 7.0],
                      rtype=F, vdict=True, extra=ex),
            ]
        out.append(_case(f"quantile_tests.cpp:125 multiple_quantile[{v.name}]", K, K10, v, V10, Kind.QUANTILE,
                         [1, 2, 3], [1.5, 4.5, 3.25, 6.0, 4.5, 7.5], rtype=F, extra=_q([0.25, 0.75])))
        k9, v9 = [1, 2, 3, 1, 2, 2, 1, 3, 2], [0, 1, 2, 3, 4, 5, 6, 7, 9]
        for interp, name, want in ((0, "LINEAR", [2.4, 4.2, 4.0]), (4, "NEAREST", [3, 4, 2]), (1, "LOWER", [0, 4, 2]),
                                   (2, "HIGHER", [3, 5, 7]), (3, "MIDPOINT", [1.5, 4.5, 4.5])):
            out.append(_case(f"quantile_tests.cpp:155 interpolation_types {name}[{v.name}]", K, k9, v, v9,
                             Kind.QUANTILE, [1, 2, 3], [float(x) for x in want], rtype=F, extra=_q([0.4], interp)))

    # ---- nunique_tests.cpp (AllTypes); bool values collapse to two
    for v in ALL_TYPES:
        is_b = v == T.BOOL8
        R = T.INT32
        out += [
            _case(f"nunique_tests.cpp:31 basic[{v.name}]", K, K10, v, V10, Kind.NUNIQUE, [1, 2, 3],
                  [2, 1, 1] if is_b else [3, 4, 3], rtype=R),
            _case(f"nunique_tests.cpp:54 empty_cols[{v.name}]", K, [], v, [], Kind.NUNIQUE, [], [], rtype=R),
            _case(f"nunique_tests.cpp:70 basic_duplicates[{v.name}]", K, K10, v, [0, 1, 2, 3, 4, 5, 3, 2, 2, 9],
                  Kind.NUNIQUE, [1, 2, 3], [2, 1, 1] if is_b else [2, 4, 1], rtype=R),
            _case(f"nunique_tests.cpp:90 zero_valid_keys[{v.name}]", K, [0, 0, 0], v, [3, 4, 5], Kind.NUNIQUE, [], [],
                  kvalid=[0, 0, 0], rtype=R),
            _case(f"nunique_tests.cpp:106 zero_valid_values[{v.name}]", K, [1, 1, 1], v, [0, 0, 0], Kind.NUNIQUE, [1],
                  [0], vvalid=[0, 0, 0], rtype=R),
            _case(f"nunique_tests.cpp:122 null_keys_and_values[{v.name}]", K, K11, v, V11, Kind.NUNIQUE,
                  [1, 2, 3, 4], [1, 1, 1, 0] if is_b else [2, 3, 2, 0], kvalid=K11_VALID, vvalid=V11_VALID_A, rtype=R),
            _case(f"nunique_tests.cpp:148 null_keys_and_values_with_duplicates[{v.name}]", K, K14, v, V14,
                  Kind.NUNIQUE, [1, 2, 3, 4], [1, 1, 1, 0] if is_b else [2, 3, 2, 0], kvalid=K14_VALID,
                  vvalid=V14_VALID_NUNIQUE, rtype=R),
            _case(f"nunique_tests.cpp:175 include_nulls[{v.name}]", K, K14, v, V14, Kind.NUNIQUE, [1, 2, 3, 4],
                  [2, 2, 1, 1] if is_b else [3, 4, 2, 1], kvalid=K14_VALID, vvalid=V14_VALID_NUNIQUE, rtype=R,
                  extra={"null_policy": NullPolicy.INCLUDE}),
        ]
        if v in INTS + FLOATS:
            out.append(_case(f"nunique_tests.cpp:202 dictionary[{v.name}]", K, [1, 2, 3, 3, 1, 2, 2, 1, 0, 3, 2, 4, 4, 2],
                             v, [0, 1, 2, 2, 3, 4, 0, 6, 7, 8, 9, 0, 0, 0], Kind.NUNIQUE, [1, 2, 3, 4], [3, 4, 2, 1],
                             kvalid=K14_VALID, vvalid=V14_VALID_NUNIQUE, rtype=R, vdict=True,
                             extra={"null_policy": NullPolicy.INCLUDE}))

    # ---- nth_element_tests.cpp (AllTypes); the result has the value's type,
    # null positions are written 0 (the reference's -1 placeholders)
    for v in ALL_TYPES:
        def nth(line, name, keys, vals, n, want, *, wvalid=None, kvalid=None, vvalid=None, policy=NullPolicy.INCLUDE,
                ekeys=(1, 2, 3)):
            if v == T.BOOL8:
                want = [int(bool(w)) for w in want]
            want = [0 if (wvalid is not None and not ok) else w for w, ok in zip(want, wvalid or [1] * len(want))]
            return _case(f"nth_element_tests.cpp:{line} {name}[{v.name}]", K, keys, v, vals, Kind.NTH_ELEMENT,
                         list(ekeys), want, evalid=wvalid, kvalid=kvalid, vvalid=vvalid, ddof=n, rtype=v,
                         extra={"null_policy": policy})
        vdup = [0, 1, 2, 3, 4, 5, 3, 2, 2, 9]
        out += [
            nth(35, "basic n=0", K10, V10, 0, [0, 1, 2]),
            nth(35, "basic n=1", K10, V10, 1, [3, 4, 7]),
            nth(35, "basic n=2", K10, V10, 2, [6, 5, 8]),
            nth(62, "empty_cols", [], [], 0, [], ekeys=()),
            nth(78, "basic_out_of_bounds", K10, vdup, 3, [0, 9, 0], wvalid=[0, 1, 0]),
            nth(94, "negative n=-1", K10, V10, -1, [6, 9, 8]),
            nth(94, "negative n=-2", K10, V10, -2, [3, 5, 7]),
            nth(94, "negative n=-3", K10, V10, -3, [0, 4, 2]),
            nth(121, "negative_out_of_bounds", K10, vdup, -4, [0, 1, 0], wvalid=[0, 1, 0]),
            nth(137, "zero_valid_keys", [1, 2, 3], [3, 4, 5], 0, [], kvalid=[0, 0, 0], ekeys=()),
            nth(153, "zero_valid_values", [1, 1, 1], [3, 4, 5], 0, [3], wvalid=[0], vvalid=[0, 0, 0], ekeys=(1,)),
            nth(169, "null_keys_and_values", K11, V11, 0, [-1, 1, 2, -1], wvalid=[0, 1, 1, 0], kvalid=K11_VALID,
                vvalid=V11_VALID_A, ekeys=(1, 2, 3, 4)),
            nth(189, "null_keys_and_values_out_of_bounds", K11, V11, 2, [6, -1, -1, -1], wvalid=[1, 0, 0, 0],
                kvalid=K11_VALID, vvalid=V11_VALID_A, ekeys=(1, 2, 3, 4)),
        ]
        for line, name, n, policy, want, wvalid in (
            (209, "exclude_nulls INCLUDE n=0", 0, NullPolicy.INCLUDE, [-1, 1, 2, 4], [0, 1, 1, 1]),
            (209, "exclude_nulls INCLUDE n=1", 1, NullPolicy.INCLUDE, [3, 4, 2, -1], [1, 1, 1, 0]),
            (209, "exclude_nulls INCLUDE n=2", 2, NullPolicy.INCLUDE, [6, -1, 8, -1], [1, 0, 1, 0]),
            (209, "exclude_nulls EXCLUDE n=0", 0, NullPolicy.EXCLUDE, [3, 1, 2, 4], None),
            (209, "exclude_nulls EXCLUDE n=1", 1, NullPolicy.EXCLUDE, [6, 4, 2, -1], [1, 1, 1, 0]),
            (209, "exclude_nulls EXCLUDE n=2", 2, NullPolicy.EXCLUDE, [-1, 9, 8, -1], [0, 1, 1, 0]),
            (251, "exclude_nulls_negative_index INCLUDE n=-1", -1, NullPolicy.INCLUDE, [6, -1, 8, -1], [1, 0, 1, 0]),
            (251, "exclude_nulls_negative_index INCLUDE n=-2", -2, NullPolicy.INCLUDE, [3, 9, 2, 4], None),
            (251, "exclude_nulls_negative_index INCLUDE n=-3", -3, NullPolicy.INCLUDE, [-1, -1, 2, -1], [0, 0, 1, 0]),
            (251, "exclude_nulls_negative_index EXCLUDE n=-1", -1, NullPolicy.EXCLUDE, [6, 9, 8, 4], None),
            (251, "exclude_nulls_negative_index EXCLUDE n=-2", -2, NullPolicy.EXCLUDE, [3, 4, 2, -1], [1, 1, 1, 0]),
            (251, "exclude_nulls_negative_index EXCLUDE n=-3", -3, NullPolicy.EXCLUDE, [-1, 1, 2, -1], [0, 1, 1, 0]),
        ):
            out.append(nth(line, name, K14, V14, n, want, wvalid=wvalid, kvalid=K14_VALID, vvalid=V14_VALID_NTH,
                           policy=policy, ekeys=(1, 2, 3, 4)))

    # ---- m2_tests.cpp (int8..int64, float, double as both key and value type)
    nan = math.nan
    for t in INTS + FLOATS:
        out += [
            _case(f"m2_tests.cpp:62 EmptyInput[{t.name}]", t, [], t, [], Kind.M2, [], [], rtype=F),
            _case(f"m2_tests.cpp:77 AllNullKeysInput[{t.name}]", t, [1, 2, 3], t, [3, 4, 5], Kind.M2, [], [],
                  kvalid=[0, 0, 0], rtype=F),
            _case(f"m2_tests.cpp:93 AllNullValuesInput[{t.name}]", t, [1, 2, 3], t, [3, 4, 5], Kind.M2, [1, 2, 3],
                  [0.0, 0.0, 0.0], vvalid=[0, 0, 0], evalid=[0, 0, 0], rtype=F),
            _case(f"m2_tests.cpp:108 SimpleInput[{t.name}]", t, K10, t, V10, Kind.M2, [1, 2, 3],
                  [18.0, 32.75, 20.0 + 2.0 / 3.0], rtype=F),
            _case(f"m2_tests.cpp:127 SimpleInputHavingNegativeValues[{t.name}]", t, K10, t,
                  [0, 1, -2, 3, -4, -5, -6, 7, -8, 9], Kind.M2, [1, 2, 3], [42.0, 122.75, 114.0], rtype=F),
            _case(f"m2_tests.cpp:146 ValuesHaveNulls[{t.name}]", t, [1, 2, 3, 4, 5, 2, 3, 2], t,
                  [0, 0, 2, 3, 0, 5, 6, 7], Kind.M2, [1, 2, 3, 4, 5], [0.0, 2.0, 8.0, 0.0, 0.0],
                  vvalid=[1, 0, 1, 1, 0, 1, 1, 1], evalid=[1, 1, 1, 1, 0], rtype=F),
            _case(f"m2_tests.cpp:162 KeysAndValuesHaveNulls[{t.name}]", t, [1, 2, 3, 1, 2, 2, 1, 0, 3, 2, 4], t,
                  [0, 1, 2, 3, 4, 0, 6, 7, 8, 9, 0], Kind.M2, [1, 2, 3, 4], [4.5, 32.0 + 2.0 / 3.0, 18.0, 0.0],
                  kvalid=[1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 1], vvalid=[0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0],
                  evalid=[1, 1, 1, 0], rtype=F),
            _case(f"m2_tests.cpp:182 InputHaveNullsAndNaNs[{t.name}]", t, [4, 3, 1, 2, 3, 1, 2, 2, 1, 0, 3, 2, 4, 4],
                  T.FLOAT64, [0.0, 0.0, 0.0, 1.0, 2.0, 3.0, 4.0, nan, 6.0, 7.0, 8.0, 9.0, 10.0, nan], Kind.M2,
                  [1, 2, 3, 4], [18.0, nan, 18.0, nan], kvalid=[1] * 9 + [0] + [1] * 4,
                  vvalid=[0, 0] + [1] * 12, rtype=F),
            _case(f"m2_tests.cpp:204 SlicedColumnsInput[{t.name}]", t,
                  [1, 2, 3, 4, 5, 1, 2, 3, 4, 5] + [4, 3, 1, 2, 3, 1, 2, 2, 1, 0, 3, 2, 4, 4]
                  + [1, 2, 3, 4, 5, 1, 2, 3, 4, 5], T.FLOAT64,
                  [3.0, 2.0, 5.0, 4.0, 6.0, 9.0, 1.0, 0.0, 1.0, 7.0]
                  + [0.0, 0.0, 0.0, 1.0, 2.0, 3.0, 4.0, nan, 6.0, 7.0, 8.0, 9.0, 10.0, nan]
                  + [9.0, 10.0, 11.0, 12.0, 0.0, 5.0, 1.0, 20.0, 19.0, 15.0], Kind.M2,
                  [1, 2, 3, 4], [18.0, nan, 18.0, nan], kvalid=[1] * 19 + [0] + [1] * 14,
                  vvalid=[1] * 10 + [0, 0] + [1] * 22, rtype=F, offset=10, size=14),
        ]
    return out


# keys_tests.cpp:199-225 expects two null-key groups ({2: 7}, {3: 7}) because the
# reference's SORTED path splits nulls by position; the hash path (this
# library and libcudf's hash groupby) groups all null keys into one group
# (nulls compare equal, hash/groupby.cu:558), so the expectation above merges
# them: null group = rows 3,4,7 -> 3+4+7 = 14.


def mismatch_case():
    """keys_tests.cpp:227-243 mismatch_num_rows: logic_error."""
    return dict(keys=[1, 2, 3], values=[0, 1, 2, 3, 4])
