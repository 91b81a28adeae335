"""Distinct rows and a distinct-key hash join through libgbx's tables, with
pylibcudf's names: distinct_count / distinct_indices / distinct
(cpp/include/cudf/stream_compaction.hpp:288-424) and distinct_hash_join's
inner and left joins (cpp/include/cudf/join.hpp:475-533)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import torch

from . import _abi, _lib
from ._abi import DuplicateKeep, NanEquality, NullEquality
from .column import Column, Table
from .groupby import TorchAllocator, _result_column

JOIN_NONE = -(2 ** 31)  # cudf::JoinNoneValue


def _stream(stream):
    return stream if stream is not None else torch.cuda.current_stream()


def distinct_count(table: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
                   allocator: Optional[TorchAllocator] = None) -> int:
    """cudf::distinct_count(table_view, null_equality): distinct rows (NaNs equal)."""
    tv, keep = table.view()
    st = _stream(stream)
    alloc = allocator if allocator is not None else TorchAllocator()
    out = C.c_int64()
    with torch.cuda.stream(st):
        _lib.check(_lib.lib().gbx_distinct_count(C.byref(tv), int(nulls_equal), C.c_void_p(st.cuda_stream),
                                                 C.byref(alloc.struct), C.byref(out)))
    return int(out.value)


def distinct_indices(table: Table, keep: DuplicateKeep = DuplicateKeep.KEEP_ANY,
                     nulls_equal: NullEquality = NullEquality.EQUAL,
                     nans_equal: NanEquality = NanEquality.ALL_EQUAL, stream=None,
                     allocator: Optional[TorchAllocator] = None) -> Column:
    """cudf::distinct_indices: INT32 row indices, one per distinct row (KEEP_NONE:
    rows whose key occurs once), in no particular order."""
    tv, keepalive = table.view()
    st = _stream(stream)
    alloc = allocator if allocator is not None else TorchAllocator()
    col = _abi.gbx_column()
    with torch.cuda.stream(st):
        _lib.check(_lib.lib().gbx_distinct_indices(C.byref(tv), int(keep), int(nulls_equal), int(nans_equal),
                                                   C.c_void_p(st.cuda_stream), C.byref(alloc.struct), C.byref(col)))
    return _result_column(col, alloc)


def gather(col: Column, indices: Column) -> Column:
    """Rows `indices` of a column (cudf::gather with in-bounds indices):
    fixed-width (a dictionary column keeps its keys), STRING (characters and
    offsets rebuilt) and STRUCT (members gathered, the struct's own mask
    kept).  Plumbing around the library's index outputs, in torch."""
    import numpy as np

    return _gather(col, np.asarray(indices.to_numpy()[0], dtype=np.int64))


def _gathered_mask(col: Column, idx, device):
    if col.mask is None:
        return None, 0
    from .column import pack_mask, unpack_mask

    valid = unpack_mask(col.mask.cpu().numpy(), col.size, col.offset)[idx]
    return torch.from_numpy(pack_mask(valid)).to(device), int(len(valid) - valid.sum())


def _gather(col: Column, idx) -> Column:
    import numpy as np

    from .column import storage_dtype

    if col.type_id == _abi.TypeId.STRUCT:
        members = [_gather(m.slice(col.offset, col.offset + col.size), idx) for m in col.children]
        device = col.mask.device if col.mask is not None else "cpu"
        mask, nulls = _gathered_mask(col, idx, device)
        return Column(_abi.TypeId.STRUCT, len(idx), None, mask, 0, nulls, children=members)
    if col.type_id == _abi.TypeId.STRING:
        offs = col.dict_keys.to_numpy()[0].astype(np.int64)[col.offset:col.offset + col.size + 1]
        starts, lens = offs[:-1][idx], (offs[1:] - offs[:-1])[idx]
        new_offs = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum(lens, out=new_offs[1:])
        total = int(new_offs[-1])
        device = col.data.device if col.data is not None else "cpu"
        pos = np.repeat(starts - new_offs[:-1], lens) + np.arange(total, dtype=np.int64)
        if total:
            chars = col.data.view(torch.uint8).index_select(0, torch.from_numpy(pos).to(device)).clone()
        else:
            chars = torch.zeros(1, dtype=torch.uint8, device=device)
        ow = np.int32 if total < 2 ** 31 else np.int64
        offsets = Column.from_numpy(new_offs.astype(ow), device=device)
        mask, nulls = _gathered_mask(col, idx, device)
        return Column(_abi.TypeId.STRING, len(idx), chars, mask, 0, nulls, dict_keys=offsets)
    device = col.data.device if col.data is not None else "cuda"
    t_idx = torch.as_tensor(idx, dtype=torch.int64, device=device)
    tid = col.index_type_id if col.type_id == _abi.TypeId.DICTIONARY32 else col.type_id
    dt = storage_dtype(tid)
    w = dt.itemsize
    data = None
    if col.data is not None and len(idx):
        elems = col.data.view(torch.uint8)[col.offset * w:(col.offset + col.size) * w].view(-1, w)
        data = elems.index_select(0, t_idx).reshape(-1).clone()
    mask, nulls = _gathered_mask(col, idx, device)
    return Column(col.type_id, len(idx), data, mask, 0, nulls, dict_keys=col.dict_keys,
                  index_type_id=col.index_type_id, scale=col.scale)


def distinct(table: Table, keys: Sequence[int], keep: DuplicateKeep = DuplicateKeep.KEEP_ANY,
             nulls_equal: NullEquality = NullEquality.EQUAL, nans_equal: NanEquality = NanEquality.ALL_EQUAL,
             stream=None) -> Table:
    """cudf::distinct(input, keys, keep, nulls_equal, nans_equal): the rows of
    `table` kept by distinct_indices over the key columns `keys`."""
    cols = table.columns()
    idx = distinct_indices(Table([cols[k] for k in keys]), keep, nulls_equal, nans_equal, stream)
    return Table([gather(c, idx) for c in cols])


def _join(build: Table, probe: Table, compare_nulls, kind, stream, allocator):
    btv, kb = build.view()
    ptv, kp = probe.view()
    st = _stream(stream)
    alloc = allocator if allocator is not None else TorchAllocator()
    bi, pi = _abi.gbx_column(), _abi.gbx_column()
    with torch.cuda.stream(st):
        _lib.check(_lib.lib().gbx_distinct_join(C.byref(btv), C.byref(ptv), int(compare_nulls), kind,
                                                C.c_void_p(st.cuda_stream), C.byref(alloc.struct), C.byref(bi),
                                                C.byref(pi)))
    return _result_column(bi, alloc), _result_column(pi, alloc)


def distinct_inner_join(build: Table, probe: Table, compare_nulls: NullEquality = NullEquality.EQUAL, stream=None,
                        allocator: Optional[TorchAllocator] = None) -> Tuple[Column, Column]:
    """distinct_hash_join(build, probe, compare_nulls).inner_join(): (build
    indices, probe indices) of the matching pairs, in no particular order."""
    return _join(build, probe, compare_nulls, 0, stream, allocator)


def distinct_left_join(build: Table, probe: Table, compare_nulls: NullEquality = NullEquality.EQUAL, stream=None,
                       allocator: Optional[TorchAllocator] = None) -> Column:
    """distinct_hash_join(...).left_join(): each probe row's build row, or
    JOIN_NONE (INT32_MIN) when it has none."""
    return _join(build, probe, compare_nulls, 1, stream, allocator)[0]
