"""Device columns and tables shaped like cudf::column_view / table_view.

A :class:`Column` holds a device buffer (a torch tensor used purely as device
memory), an optional cudf-layout validity bitmask (32-bit words, bit i of word
i//32 set when row i is valid), a row offset, and for DICTIONARY32 columns the
dictionary's keys column.  PyTorch only provides memory and streams here; all
groupby work runs in libgbx's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from ._abi import TYPE_WIDTH, TypeId, gbx_column_view, gbx_table_view

_NP_TO_TYPE = {
    np.dtype(np.int8): TypeId.INT8,
    np.dtype(np.int16): TypeId.INT16,
    np.dtype(np.int32): TypeId.INT32,
    np.dtype(np.int64): TypeId.INT64,
    np.dtype(np.uint8): TypeId.UINT8,
    np.dtype(np.uint16): TypeId.UINT16,
    np.dtype(np.uint32): TypeId.UINT32,
    np.dtype(np.uint64): TypeId.UINT64,
    np.dtype(np.float32): TypeId.FLOAT32,
    np.dtype(np.float64): TypeId.FLOAT64,
    np.dtype(np.bool_): TypeId.BOOL8,
}

# storage dtype of each fixed-width type id
_STORAGE = {
    TypeId.INT8: np.int8, TypeId.INT16: np.int16, TypeId.INT32: np.int32, TypeId.INT64: np.int64,
    TypeId.UINT8: np.uint8, TypeId.UINT16: np.uint16, TypeId.UINT32: np.uint32, TypeId.UINT64: np.uint64,
    TypeId.FLOAT32: np.float32, TypeId.FLOAT64: np.float64, TypeId.BOOL8: np.uint8,
    TypeId.TIMESTAMP_DAYS: np.int32, TypeId.TIMESTAMP_SECONDS: np.int64,
    TypeId.TIMESTAMP_MILLISECONDS: np.int64, TypeId.TIMESTAMP_MICROSECONDS: np.int64,
    TypeId.TIMESTAMP_NANOSECONDS: np.int64,
    TypeId.DURATION_DAYS: np.int32, TypeId.DURATION_SECONDS: np.int64,
    TypeId.DURATION_MILLISECONDS: np.int64, TypeId.DURATION_MICROSECONDS: np.int64,
    TypeId.DURATION_NANOSECONDS: np.int64,
    TypeId.DECIMAL32: np.int32, TypeId.DECIMAL64: np.int64,
}


def storage_dtype(type_id: int) -> np.dtype:
    return np.dtype(_STORAGE[TypeId(type_id)])


def type_of(arr: np.ndarray) -> TypeId:
    return _NP_TO_TYPE[arr.dtype]


def pack_mask(valid: np.ndarray) -> np.ndarray:
    """Bool array -> cudf bitmask words (int32, LSB-first), padded to 64 bytes."""
    valid = np.asarray(valid, dtype=bool)
    nbytes = ((len(valid) + 511) // 512) * 64
    packed = np.packbits(valid, bitorder="little")
    buf = np.zeros(max(nbytes, 64), dtype=np.uint8)
    buf[: len(packed)] = packed
    return buf.view(np.int32)


def unpack_mask(words: np.ndarray, n: int, offset: int = 0) -> np.ndarray:
    bits = np.unpackbits(np.asarray(words).view(np.uint8), bitorder="little")
    return bits[offset: offset + n].astype(bool)


def _to_device(arr: np.ndarray, device, pin: bool = False) -> torch.Tensor:
    t = torch.from_numpy(np.ascontiguousarray(arr))
    if pin:
        t = t.pin_memory()
    return t.to(device, non_blocking=pin)


class Column:
    """A borrowed-or-owned device column (cudf::column_view)."""

    def __init__(
        self,
        type_id: int,
        size: int,
        data: Optional[torch.Tensor],
        mask: Optional[torch.Tensor] = None,
        offset: int = 0,
        null_count: Optional[int] = None,
        dict_keys: Optional["Column"] = None,
        index_type_id: int = TypeId.INT32,
        scale: int = 0,
        children: Optional[Sequence["Column"]] = None,
    ):
        self.type_id = TypeId(type_id)
        self.children = list(children) if children is not None else []
        self.size = int(size)
        self.data = data
        self.mask = mask
        self.offset = int(offset)
        self._null_count = null_count if mask is not None else 0
        self.dict_keys = dict_keys
        self.index_type_id = TypeId(index_type_id)
        self.scale = int(scale)
        self._view = None

    # ---- construction
    @classmethod
    def from_numpy(cls, values: np.ndarray, valid: Optional[np.ndarray] = None, type_id: Optional[int] = None,
                   device="cuda", scale: int = 0, pin: bool = False) -> "Column":
        values = np.asarray(values)
        tid = TypeId(type_id) if type_id is not None else type_of(values)
        if tid == TypeId.BOOL8:
            values = values.astype(np.uint8)
        else:
            values = values.astype(storage_dtype(tid), copy=False)
        data = _to_device(values, device, pin) if len(values) else None
        mask = None
        nulls = 0
        if valid is not None:
            valid = np.asarray(valid, dtype=bool)
            nulls = int(len(valid) - valid.sum())
            mask = _to_device(pack_mask(valid), device, pin)
        return cls(tid, len(values), data, mask, 0, nulls, scale=scale)

    @classmethod
    def dictionary(cls, indices: "Column", keys: "Column", mask: Optional[torch.Tensor] = None,
                   null_count: Optional[int] = None) -> "Column":
        """DICTIONARY32 column: `indices` (integer) into `keys`."""
        return cls(TypeId.DICTIONARY32, indices.size, indices.data, mask if mask is not None else indices.mask,
                   indices.offset, null_count if mask is not None else indices._null_count,
                   dict_keys=keys, index_type_id=indices.type_id)

    @classmethod
    def from_strings(cls, values, valid: Optional[np.ndarray] = None, device="cuda") -> "Column":
        """STRING column: UTF-8 characters in `data`, an INT32 offsets child
        (held in `dict_keys`, as the C ABI passes it) and an optional mask
        (None entries of `values` are nulls too)."""
        vals = list(values)
        ok = np.array([v is not None for v in vals], dtype=bool)
        if valid is not None:
            ok &= np.asarray(valid, dtype=bool)
        enc = [(v if v is not None else "").encode("utf-8") for v in vals]
        lens = np.array([len(b) for b in enc], dtype=np.int64)
        offs = np.zeros(len(vals) + 1, dtype=np.int64)
        np.cumsum(lens, out=offs[1:])
        ow = np.int32 if offs[-1] < 2 ** 31 else np.int64
        chars = np.frombuffer(b"".join(enc), dtype=np.uint8).copy() if offs[-1] else np.zeros(1, np.uint8)
        offsets = cls.from_numpy(offs.astype(ow), device=device)
        data = _to_device(chars, device, False)
        mask = None
        nulls = 0
        if not ok.all():
            nulls = int(len(ok) - ok.sum())
            mask = _to_device(pack_mask(ok), device, False)
        return cls(TypeId.STRING, len(vals), data, mask, 0, nulls, dict_keys=offsets)

    @classmethod
    def struct(cls, members: Sequence["Column"], valid: Optional[np.ndarray] = None, device="cuda") -> "Column":
        """STRUCT column of `members` (equal sizes; fixed-width, STRING or
        STRUCT), with an optional validity of its own."""
        members = list(members)
        n = members[0].size if members else 0
        mask = None
        nulls = 0
        if valid is not None:
            valid = np.asarray(valid, dtype=bool)
            nulls = int(len(valid) - valid.sum())
            mask = _to_device(pack_mask(valid), device, False)
        return cls(TypeId.STRUCT, n, None, mask, 0, nulls, children=members)

    def slice(self, begin: int, end: int) -> "Column":
        """A view of rows [begin, end) sharing this column's buffers (cudf::slice)."""
        return Column(self.type_id, end - begin, self.data, self.mask, self.offset + begin, None,
                      self.dict_keys, self.index_type_id, self.scale, self.children)

    # ---- properties
    @property
    def null_count(self) -> int:
        if self.mask is None:
            return 0
        if self._null_count is None:
            valid = unpack_mask(self.mask.cpu().numpy(), self.size, self.offset)
            self._null_count = int(self.size - valid.sum())
        return self._null_count

    def has_nulls(self) -> bool:
        return self.null_count > 0

    def view(self) -> gbx_column_view:
        v = gbx_column_view()
        v.type_id = int(self.type_id)
        v.scale = self.scale
        v.size = self.size
        v.offset = self.offset
        v.data = self.data.data_ptr() if self.data is not None else None
        v.null_mask = self.mask.data_ptr() if self.mask is not None else None
        v.null_count = -1 if (self.mask is not None and self._null_count is None) else int(self._null_count or 0)
        v.index_type_id = int(self.index_type_id) if self.type_id == TypeId.DICTIONARY32 else 0
        if self.dict_keys is not None:
            self._kview = self.dict_keys.view()
            v.dict_keys = C.pointer(self._kview)
        if self.type_id == TypeId.STRUCT:
            # the members' views, as an array the view points at
            self._members = (gbx_column_view * max(1, len(self.children)))()
            for i, m in enumerate(self.children):
                self._members[i] = m.view()
            v.num_children = len(self.children)
            v.dict_keys = C.cast(self._members, C.POINTER(gbx_column_view))
        self._view = v
        return v

    # ---- host conversion
    def to_numpy(self):
        """(values, valid) on the host; valid is None when the column has no mask.
        A STRING column's values are a numpy object array of str; a STRUCT
        column's values are the list of its members' (values, valid) over
        this column's rows."""
        if self.type_id == TypeId.STRUCT:
            vals = [m.slice(self.offset, self.offset + self.size).to_numpy() for m in self.children]
            valid = None
            if self.mask is not None:
                valid = unpack_mask(self.mask.detach().cpu().numpy(), self.size, self.offset)
            return vals, valid
        if self.type_id == TypeId.STRING:
            offs = self.dict_keys.to_numpy()[0].astype(np.int64)
            raw = self.data.detach().cpu().numpy().view(np.uint8).tobytes() if self.data is not None else b""
            o = offs[self.offset: self.offset + self.size + 1]
            vals = np.array([raw[o[i]:o[i + 1]].decode("utf-8") for i in range(self.size)], dtype=object)
            valid = None
            if self.mask is not None:
                valid = unpack_mask(self.mask.detach().cpu().numpy(), self.size, self.offset)
            return vals, valid
        if self.type_id == TypeId.DICTIONARY32:
            dt = storage_dtype(self.index_type_id)
        else:
            dt = storage_dtype(self.type_id)
        if self.size == 0 or self.data is None:
            vals = np.zeros(0, dtype=dt)
        else:
            raw = self.data.detach().cpu().numpy().view(np.uint8)
            w = dt.itemsize
            vals = raw[self.offset * w: (self.offset + self.size) * w].view(dt).copy()
        if self.type_id == TypeId.BOOL8:
            vals = vals.astype(bool)
        valid = None
        if self.mask is not None:
            valid = unpack_mask(self.mask.detach().cpu().numpy(), self.size, self.offset)
        return vals, valid

    def __len__(self):
        return self.size

    def __repr__(self):
        return f"Column({self.type_id.name}, size={self.size}, nulls={self._null_count})"


class Table:
    """An ordered set of equal-length columns (cudf::table_view)."""

    def __init__(self, columns: Sequence[Column]):
        self._columns = list(columns)

    def columns(self):
        return list(self._columns)

    def num_columns(self) -> int:
        return len(self._columns)

    def num_rows(self) -> int:
        return self._columns[0].size if self._columns else 0

    def view(self):
        arr = (gbx_column_view * max(1, len(self._columns)))()
        for i, c in enumerate(self._columns):
            arr[i] = c.view()
        tv = gbx_table_view()
        tv.num_columns = len(self._columns)
        tv.columns = C.cast(arr, C.POINTER(gbx_column_view))
        tv._keep = arr
        return tv, arr

    def __getitem__(self, i):
        return self._columns[i]

    def __len__(self):
        return len(self._columns)
