"""Python wrapper of the CPU oracle (oracle/gbx_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the parity checker.  The product (libgbx /
cudf_b200) never imports it.

Columns are given as :class:`HostCol` (numpy values + optional bool validity);
the oracle returns numpy arrays in first-occurrence group order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from cudf_b200._abi import TypeId, aggregation_array, gbx_aggregation, gbx_column_view, gbx_request, gbx_table_view
from cudf_b200.column import pack_mask, storage_dtype, type_of

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libgbx_oracle.so")


def build() -> str:
    src = [os.path.join(HERE, f) for f in ("gbx_oracle.c", "gbx_oracle.h", "Makefile")]
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


class gbo_column(C.Structure):
    _fields_ = [
        ("type_id", C.c_int32),
        ("scale", C.c_int32),
        ("size", C.c_int64),
        ("data", C.c_void_p),
        ("valid", C.POINTER(C.c_uint8)),
        ("str_offsets", C.POINTER(C.c_int64)),
    ]


class gbo_result(C.Structure):
    _fields_ = [
        ("num_groups", C.c_int64),
        ("num_key_columns", C.c_int32),
        ("num_requests", C.c_int32),
        ("keys", C.POINTER(gbo_column)),
        ("num_results", C.POINTER(C.c_int32)),
        ("results", C.POINTER(C.POINTER(gbo_column))),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        h = C.CDLL(build())
        h.gbo_groupby.restype = C.c_int
        h.gbo_groupby.argtypes = [C.POINTER(gbx_table_view), C.c_int32, C.POINTER(gbx_request), C.c_int32,
                                  C.c_int32, C.POINTER(C.POINTER(gbo_result))]
        h.gbo_result_free.restype = None
        h.gbo_result_free.argtypes = [C.POINTER(gbo_result)]
        h.gbo_last_error.restype = C.c_char_p
        h.gbo_target_type.restype = C.c_int32
        h.gbo_target_type.argtypes = [C.c_int32, C.c_int32]
        _lib = h
    return _lib


@dataclass
class HostCol:
    """A host column: values (storage dtype), optional validity, optional
    dictionary keys (then `values` are the integer indices)."""

    values: np.ndarray
    valid: Optional[np.ndarray] = None
    type_id: Optional[int] = None
    scale: int = 0
    dict_keys: Optional["HostCol"] = None
    offset: int = 0
    size: Optional[int] = None
    children: Optional[list] = None  # STRUCT: member HostCols (row r is row offset + r of each)
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        if self.type_id == TypeId.STRUCT:
            n = self.children[0].size if self.children else 0
            self.values = np.zeros(0, dtype=np.uint8)
            if self.valid is not None:
                self.valid = np.asarray(self.valid, dtype=bool)
            if self.size is None:
                self.size = n - self.offset
            return
        if self.type_id == TypeId.STRING:
            # str (or None: null) values; UTF-8 characters and int64 offsets for the view
            self.values = np.array(list(self.values), dtype=object)
            ok = np.array([v is not None for v in self.values], dtype=bool)
            if self.valid is not None:
                ok &= np.asarray(self.valid, dtype=bool)
            self.valid = None if ok.all() else ok
            enc = [(v if v is not None else "").encode("utf-8") for v in self.values]
            offs = np.zeros(len(enc) + 1, dtype=np.int64)
            np.cumsum([len(b) for b in enc], out=offs[1:])
            self._chars = np.frombuffer(b"".join(enc) or b"\0", dtype=np.uint8).copy()
            self.dict_keys = HostCol(offs)
            if self.size is None:
                self.size = len(self.values) - self.offset
            return
        self.values = np.asarray(self.values)
        if self.dict_keys is not None:
            self.type_id = TypeId.DICTIONARY32
        elif self.type_id is None:
            self.type_id = type_of(self.values)
        if self.type_id == TypeId.BOOL8:
            self.values = self.values.astype(np.uint8)
        elif self.type_id != TypeId.DICTIONARY32:
            self.values = np.ascontiguousarray(self.values.astype(storage_dtype(self.type_id), copy=False))
        if self.valid is not None:
            self.valid = np.asarray(self.valid, dtype=bool)
        if self.size is None:
            self.size = len(self.values) - self.offset

    @property
    def index_type(self) -> int:
        return type_of(self.values) if self.type_id == TypeId.DICTIONARY32 else 0

    def view(self) -> gbx_column_view:
        v = gbx_column_view()
        v.type_id = int(self.type_id)
        v.scale = self.scale
        v.size = self.size
        v.offset = self.offset
        if self.type_id == TypeId.STRUCT:
            vals = np.zeros(0, dtype=np.uint8)
            members = (gbx_column_view * max(1, len(self.children)))()
            for i, m in enumerate(self.children):
                members[i] = m.view()
            v.num_children = len(self.children)
            v.dict_keys = C.cast(members, C.POINTER(gbx_column_view))
            self._members = members
        elif self.type_id == TypeId.STRING:
            vals = self._chars
        else:
            vals = np.ascontiguousarray(self.values)
        self._keep = [vals]
        v.data = vals.ctypes.data if len(vals) else None
        if self.valid is not None:
            m = pack_mask(self.valid)
            self._keep.append(m)
            v.null_mask = m.ctypes.data
            v.null_count = -1
        else:
            v.null_mask = None
            v.null_count = 0
        if self.dict_keys is not None:
            kv = self.dict_keys.view()
            self._keep.append(kv)
            v.dict_keys = C.pointer(kv)
            v.index_type_id = int(self.index_type) if self.type_id == TypeId.DICTIONARY32 else 0
        return v


def _np_of(col: gbo_column, n: int) -> Tuple[int, np.ndarray, Optional[np.ndarray]]:
    tid = TypeId(col.type_id)
    if tid == TypeId.STRING:
        offs = np.ctypeslib.as_array(col.str_offsets, shape=(n + 1,)).copy() if col.str_offsets else np.zeros(1, np.int64)
        raw = bytes((C.c_uint8 * int(offs[-1])).from_address(col.data)) if offs[-1] else b""
        vals = np.array([raw[offs[i]:offs[i + 1]].decode("utf-8") for i in range(n)], dtype=object)
        valid = None
        if col.valid:
            valid = np.ctypeslib.as_array(col.valid, shape=(n,)).astype(bool).copy() if n else np.zeros(0, bool)
        return int(tid), vals, valid
    dt = np.dtype(np.int32) if tid == TypeId.DICTIONARY32 else storage_dtype(tid)
    if n == 0 or not col.data:
        vals = np.zeros(0, dtype=dt)
    else:
        buf = (C.c_uint8 * (n * dt.itemsize)).from_address(col.data)
        vals = np.frombuffer(bytes(buf), dtype=dt).copy()
    if tid == TypeId.BOOL8:
        vals = vals.astype(bool)
    valid = None
    if col.valid:
        valid = np.ctypeslib.as_array(col.valid, shape=(n,)).astype(bool).copy() if n else np.zeros(0, bool)
    return int(tid), vals, valid


def groupby(keys: Sequence[HostCol], requests: Sequence[Tuple[HostCol, Sequence[Tuple[int, int]]]],
            null_policy: int = 0, threads: int = 1) -> dict:
    """Runs the oracle.  `requests` is [(values, [(kind, ddof[, extra]), ...]), ...]
    (extra: a dict of null_policy / interpolation / quantiles, as
    cudf_b200._abi.fill_aggregation reads it).

    Returns {"num_groups", "keys": [(type_id, values, valid)], "results": [[(type_id, values, valid)]]}.
    Raises RuntimeError carrying the gbx_status on invalid input."""
    kviews = (gbx_column_view * max(1, len(keys)))()
    for i, k in enumerate(keys):
        kviews[i] = k.view()
    tv = gbx_table_view()
    tv.num_columns = len(keys)
    tv.columns = C.cast(kviews, C.POINTER(gbx_column_view))
    reqs = (gbx_request * max(1, len(requests)))()
    keep = []
    for i, (vals, aggs) in enumerate(requests):
        reqs[i].values = vals.view()
        arr, kept = aggregation_array(aggs)
        keep.append(kept)
        reqs[i].num_aggregations = len(aggs)
        reqs[i].aggregations = C.cast(arr, C.POINTER(gbx_aggregation))
    out = C.POINTER(gbo_result)()
    st = lib().gbo_groupby(C.byref(tv), int(null_policy), reqs, len(requests), int(threads), C.byref(out))
    if st != 0:
        err = RuntimeError(lib().gbo_last_error().decode())
        err.status = st
        raise err
    try:
        r = out.contents
        n = r.num_groups
        res = {"num_groups": n, "keys": [], "results": []}
        for c in range(r.num_key_columns):
            res["keys"].append(_np_of(r.keys[c], n))
        for q in range(r.num_requests):
            # a QUANTILE column holds num_quantiles rows per group
            res["results"].append([_np_of(r.results[q][k], r.results[q][k].size) for k in range(r.num_results[q])])
        return res
    finally:
        lib().gbo_result_free(out)


def target_type(type_id: int, kind: int) -> int:
    return lib().gbo_target_type(int(type_id), int(kind))
