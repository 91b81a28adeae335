"""Hash joins with pylibcudf.join's shape (cudf::inner_join / left_join /
full_join / left_semi_join / left_anti_join, join.hpp:107-260), on libgbx's
gbx_hash_join.  Gather maps come back as INT32 columns in no particular order;
a row without a match on the other side is JOIN_NONE (INT32_MIN,
cudf::JoinNoneValue)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import torch

from . import _abi, _lib
from ._abi import JoinKind, NullEquality
from .column import Column, Table
from .groupby import TorchAllocator, _result_column
from .stream_compaction import JOIN_NONE, _stream  # noqa: F401


def _hash_join(left: Table, right: Table, nulls_equal, kind, stream, allocator):
    ltv, kl = left.view()
    rtv, kr = right.view()
    st = _stream(stream)
    alloc = allocator if allocator is not None else TorchAllocator()
    li, ri = _abi.gbx_column(), _abi.gbx_column()
    with torch.cuda.stream(st):
        _lib.check(_lib.lib().gbx_hash_join(C.byref(ltv), C.byref(rtv), int(nulls_equal), int(kind),
                                            C.c_void_p(st.cuda_stream), C.byref(alloc.struct), C.byref(li),
                                            C.byref(ri)))
    return _result_column(li, alloc), _result_column(ri, alloc)


def inner_join(left_keys: Table, right_keys: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
               allocator: Optional[TorchAllocator] = None) -> Tuple[Column, Column]:
    """(left rows, right rows) of every matching pair."""
    return _hash_join(left_keys, right_keys, nulls_equal, JoinKind.INNER, stream, allocator)


def left_join(left_keys: Table, right_keys: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
              allocator: Optional[TorchAllocator] = None) -> Tuple[Column, Column]:
    """Every left row with each matching right row, or JOIN_NONE."""
    return _hash_join(left_keys, right_keys, nulls_equal, JoinKind.LEFT, stream, allocator)


def full_join(left_keys: Table, right_keys: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
              allocator: Optional[TorchAllocator] = None) -> Tuple[Column, Column]:
    """The left join's pairs, then (JOIN_NONE, right row) for each unmatched
    right row."""
    return _hash_join(left_keys, right_keys, nulls_equal, JoinKind.FULL, stream, allocator)


def left_semi_join(left_keys: Table, right_keys: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
                   allocator: Optional[TorchAllocator] = None) -> Column:
    """The left rows that have a match."""
    return _hash_join(left_keys, right_keys, nulls_equal, JoinKind.LEFT_SEMI, stream, allocator)[0]


def left_anti_join(left_keys: Table, right_keys: Table, nulls_equal: NullEquality = NullEquality.EQUAL, stream=None,
                   allocator: Optional[TorchAllocator] = None) -> Column:
    """The left rows that have no match."""
    return _hash_join(left_keys, right_keys, nulls_equal, JoinKind.LEFT_ANTI, stream, allocator)[0]
