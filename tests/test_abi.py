"""CPU tests of the drop-in boundary: libgbx.so loads and exports every entry
point include/gbx.h declares, the ctypes mirror matches the C layout, the
target-type table matches the oracle's restatement, and host-side validation
(which runs before any CUDA call) behaves like the reference's CUDF_EXPECTS."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from cudf_b200 import _abi, _lib
from cudf_b200._abi import Kind, TypeId
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gbx.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"GBX_API\s+[\w\s\*]+?\b(gbx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), f"{n} missing from libgbx.so"
        assert n in _abi.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.gbx_abi_version() == 5


STRUCTS = ["gbx_column_view", "gbx_table_view", "gbx_aggregation", "gbx_request", "gbx_allocator",
           "gbx_column", "gbx_aggregation_result", "gbx_result", "gbx_stats", "gbx_batch_instance",
           "gbx_batch_options", "gbx_batch_output", "gbx_batch_stats", "gbx_server_options", "gbx_server_timing",
           "gbx_server_stats"]


def test_ctypes_layout_matches_c_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for s in STRUCTS:
        ct = getattr(_abi, s)
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{s}.{fname} %zu\\n", offsetof({s}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c_layout = dict(l.rsplit(" ", 1) for l in out if l)
    for s in STRUCTS:
        ct = getattr(_abi, s)
        assert int(c_layout[s]) == C.sizeof(ct), s
        for fname, _ in ct._fields_:
            assert int(c_layout[f"{s}.{fname}"]) == getattr(ct, fname).offset, f"{s}.{fname}"


def test_target_types_match_oracle():
    lib = _lib.lib()
    computed = {Kind.SUM, Kind.PRODUCT, Kind.MIN, Kind.MAX, Kind.COUNT_VALID, Kind.COUNT_ALL,
                Kind.SUM_OF_SQUARES, Kind.MEAN, Kind.VARIANCE, Kind.STD, Kind.ARGMIN, Kind.ARGMAX,
                Kind.M2, Kind.MEDIAN, Kind.QUANTILE, Kind.NUNIQUE, Kind.NTH_ELEMENT}
    for t in TypeId:
        for k in Kind:
            want = orc.target_type(t, k) if k in computed else 0
            assert lib.gbx_target_type(int(t), int(k)) == want, (t.name, k.name)


def _keys_view(n=3):
    arr = np.arange(n, dtype=np.int32)
    cv = _abi.gbx_column_view()
    cv.type_id = TypeId.INT32
    cv.size = n
    cv.data = arr.ctypes.data  # never dereferenced: validation fails first
    cols = (_abi.gbx_column_view * 1)(cv)
    tv = _abi.gbx_table_view(1, 0, C.cast(cols, C.POINTER(_abi.gbx_column_view)))
    return tv, (arr, cols)


def _request(n, kind):
    r = _abi.gbx_request()
    r.values.type_id = TypeId.INT32
    r.values.size = n
    aggs = (_abi.gbx_aggregation * 1)()
    aggs[0].kind = int(kind)
    r.num_aggregations = 1
    r.aggregations = C.cast(aggs, C.POINTER(_abi.gbx_aggregation))
    return r, aggs


def test_size_mismatch_is_logic_error():
    """keys_tests.cpp:227-243 / groupby.cu:210-214."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == 0
    r, keep2 = _request(5, Kind.COUNT_VALID)
    out = C.POINTER(_abi.gbx_result)()
    st = lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out))
    assert st == _abi.Status.ERR_LOGIC
    assert b"Size mismatch" in lib.gbx_last_error()
    with pytest.raises(_lib.LogicError):
        _lib.check(st)
    lib.gbx_groupby_destroy(h)


@pytest.mark.parametrize("vtype", [TypeId.STRING, TypeId.STRUCT, TypeId.LIST, TypeId.DECIMAL128])
def test_values_only_counted(vtype):
    """STRING / STRUCT / LIST / DECIMAL128 values: COUNT is computed (through
    a stand-in, on the device), and MIN / MAX of strings; any other kind is
    UNSUPPORTED before device work; the no-allocation entry point refuses
    them all."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == 0
    for kind in (Kind.SUM, Kind.MIN, Kind.MEAN):
        r, keep2 = _request(3, kind)
        r.values.type_id = int(vtype)
        out = C.POINTER(_abi.gbx_result)()
        st = lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out))
        if vtype == TypeId.STRING and kind == Kind.MIN:
            # MIN / MAX of strings are computed; this view lacks its offsets
            assert st == _abi.Status.ERR_LOGIC and b"offsets" in lib.gbx_last_error()
        else:
            assert st == _abi.Status.ERR_UNSUPPORTED
    r, keep2 = _request(3, Kind.COUNT_VALID)
    r.values.type_id = int(vtype)
    res = (_abi.gbx_column * 1)()
    ng = C.c_int64()
    assert lib.gbx_groupby_aggregate_noalloc(h, C.byref(r), 1, None, None, res, 8, C.byref(ng)) == \
        _abi.Status.ERR_UNSUPPORTED
    lib.gbx_groupby_destroy(h)


def test_string_extremes_with_sorted_keys_refused():
    """MIN / MAX of strings run on unsorted keys only."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 1, C.byref(h)) == 0
    offs = np.array([0, 1, 2, 3], np.int32)
    chars = np.frombuffer(b"abc", np.uint8).copy()
    ov = _abi.gbx_column_view()
    ov.type_id = TypeId.INT32
    ov.size = 4
    ov.data = offs.ctypes.data
    r, keep2 = _request(3, Kind.MAX)
    r.values.type_id = int(TypeId.STRING)
    r.values.data = chars.ctypes.data
    r.values.dict_keys = C.pointer(ov)
    out = C.POINTER(_abi.gbx_result)()
    assert lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out)) == _abi.Status.ERR_UNSUPPORTED
    assert b"sorted" in lib.gbx_last_error()
    lib.gbx_groupby_destroy(h)


@pytest.mark.parametrize("kind", [Kind.ANY, Kind.ALL, 19, 30])
def test_kinds_not_computed_are_reported(kind):
    """ANY / ALL and libcudf's later kinds (ROW_NUMBER onwards) are not
    computed here: UNSUPPORTED, before any device work."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == 0
    r, keep2 = _request(3, kind)
    out = C.POINTER(_abi.gbx_result)()
    assert lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out)) == _abi.Status.ERR_UNSUPPORTED
    assert lib.gbx_can_use_hash_groupby(C.byref(r), 1) == 0
    lib.gbx_groupby_destroy(h)


@pytest.mark.parametrize("kind", [Kind.M2, Kind.MEDIAN, Kind.QUANTILE, Kind.NUNIQUE, Kind.NTH_ELEMENT])
def test_sort_path_kinds_are_not_hash_kinds(kind):
    """can_use_hash_groupby (hash/groupby.cu:635-651) is false for the sort
    path's kinds, which gbx_groupby_aggregate computes all the same."""
    lib = _lib.lib()
    r, keep = _request(3, kind)
    assert lib.gbx_can_use_hash_groupby(C.byref(r), 1) == 0
    assert lib.gbx_target_type(int(TypeId.INT32), int(kind)) != 0


def _aggregate_status(agg_fields):
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == 0
    r, aggs = _request(3, agg_fields.pop("kind"))
    for f, v in agg_fields.items():
        setattr(aggs[0], f, v)
    out = C.POINTER(_abi.gbx_result)()
    st = lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out))
    msg = lib.gbx_last_error()
    lib.gbx_groupby_destroy(h)
    return st, msg


def test_quantile_arguments_are_checked():
    """A QUANTILE without its array, or with an interpolation outside
    cudf::interpolation, is a logic error before any device work."""
    st, msg = _aggregate_status({"kind": Kind.QUANTILE, "num_quantiles": 2})
    assert st == _abi.Status.ERR_LOGIC and b"quantile array" in msg
    st, msg = _aggregate_status({"kind": Kind.QUANTILE, "interpolation": 7})
    assert st == _abi.Status.ERR_LOGIC and b"interpolation" in msg
    st, msg = _aggregate_status({"kind": Kind.NUNIQUE, "null_policy": 3})
    assert st == _abi.Status.ERR_LOGIC and b"null_policy" in msg


def test_invalid_type_agg_combination_is_logic_error():
    """VAR of a timestamp column: no target type (aggregation.hpp:1212-1335)."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == 0
    r, keep2 = _request(3, Kind.VARIANCE)
    r.values.type_id = TypeId.TIMESTAMP_DAYS
    out = C.POINTER(_abi.gbx_result)()
    assert lib.gbx_groupby_aggregate(h, C.byref(r), 1, None, None, C.byref(out)) == _abi.Status.ERR_LOGIC
    assert lib.gbx_can_use_hash_groupby(C.byref(r), 1) == 0
    lib.gbx_groupby_destroy(h)


def test_create_checks_key_columns_and_policy():
    """A STRING key needs its offsets child; list / struct keys are refused."""
    lib = _lib.lib()
    tv, keep = _keys_view(3)
    h = C.c_void_p()
    assert lib.gbx_groupby_create(C.byref(tv), 7, 0, C.byref(h)) == _abi.Status.ERR_LOGIC
    keep[1][0].type_id = TypeId.STRING
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.ERR_LOGIC
    assert b"offsets" in lib.gbx_last_error()
    offs = np.array([0, 1, 2, 3], dtype=np.int32)
    ov = _abi.gbx_column_view()
    ov.type_id = TypeId.INT32
    ov.size = 4
    ov.data = offs.ctypes.data
    keep[1][0].dict_keys = C.pointer(ov)
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.OK
    lib.gbx_groupby_destroy(h)
    keep[1][0].type_id = TypeId.LIST
    assert lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)) == _abi.Status.ERR_UNSUPPORTED


def test_can_use_hash_groupby_for_hash_kinds():
    lib = _lib.lib()
    for k in (Kind.SUM, Kind.MIN, Kind.MAX, Kind.COUNT_VALID, Kind.MEAN, Kind.VARIANCE, Kind.STD, Kind.ARGMIN,
              Kind.ARGMAX):
        r, keep = _request(3, k)
        assert lib.gbx_can_use_hash_groupby(C.byref(r), 1) == 1


# ---- batched form: schema checks run on the host before any CUDA call

def _batch_instance(n, key_type=TypeId.INT32, kind=Kind.SUM, value_type=TypeId.INT32):
    tv, keep = _keys_view(n)
    keep[1][0].type_id = key_type
    r, aggs = _request(n, kind)
    r.values.type_id = value_type
    reqs = (_abi.gbx_request * 1)(r)
    inst = _abi.gbx_batch_instance(tv, C.cast(reqs, C.POINTER(_abi.gbx_request)))
    return inst, (tv, keep, r, aggs, reqs)


def _create_batch(insts, nreq=1, opts=None):
    arr = (_abi.gbx_batch_instance * max(1, len(insts)))(*insts)
    h = C.c_void_p()
    o = opts if opts is not None else _abi.gbx_batch_options()
    st = _lib.lib().gbx_batch_create(arr, len(insts), nreq, C.byref(o), None, None, C.byref(h))
    return st, _lib.lib().gbx_last_error()


def test_batch_needs_instances_of_one_schema():
    a, ka = _batch_instance(4)
    b, kb = _batch_instance(9, key_type=TypeId.INT64)
    st, msg = _create_batch([a, b])
    assert st == _abi.Status.ERR_LOGIC and b"key column 0 differs" in msg
    c, kc = _batch_instance(9, kind=Kind.MAX)
    st, msg = _create_batch([a, c])
    assert st == _abi.Status.ERR_LOGIC and b"differs in aggregations" in msg
    d, kd = _batch_instance(9, value_type=TypeId.INT64)
    st, msg = _create_batch([a, d])
    assert st == _abi.Status.ERR_LOGIC and b"values differ in type" in msg


def test_batch_rejects_bad_arguments():
    a, ka = _batch_instance(4)
    st, _ = _create_batch([])
    assert st == _abi.Status.ERR_LOGIC
    st, _ = _create_batch([a], opts=_abi.gbx_batch_options(block_threads=300))
    assert st == _abi.Status.ERR_LOGIC
    st, _ = _create_batch([a], opts=_abi.gbx_batch_options(null_policy=5))
    assert st == _abi.Status.ERR_LOGIC
    st, _ = _create_batch([a], opts=_abi.gbx_batch_options(force_mode=9))
    assert st == _abi.Status.ERR_LOGIC
    # a request whose values are shorter than the keys (groupby.cu:210-214)
    b, kb = _batch_instance(4)
    kb[4][0].values.size = 3
    st, msg = _create_batch([a, b])
    assert st == _abi.Status.ERR_LOGIC and b"Size mismatch" in msg


def test_batch_rejects_dictionary_keys_and_sort_kinds():
    a, ka = _batch_instance(4, key_type=TypeId.DICTIONARY32)
    st, _ = _create_batch([a])
    assert st == _abi.Status.ERR_UNSUPPORTED
    b, kb = _batch_instance(4, kind=Kind.MEDIAN)
    st, _ = _create_batch([b])
    assert st == _abi.Status.ERR_UNSUPPORTED


def test_batch_rejects_argmin_argmax():
    """The batched kernels address rows within their instance, so the row
    indices ARGMIN/ARGMAX return are left to the plain form."""
    for kind in (Kind.ARGMIN, Kind.ARGMAX):
        a, ka = _batch_instance(4, kind=kind)
        st, msg = _create_batch([a])
        assert st == _abi.Status.ERR_UNSUPPORTED and b"batched form" in msg
