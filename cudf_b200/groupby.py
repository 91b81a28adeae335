"""Hash groupby-aggregation, shaped like pylibcudf.groupby
(python/cudf/cudf/_lib/pylibcudf/groupby.pyx:84-181) over libgbx's C ABI.

    gb = GroupBy(Table([keys]), null_handling=NullPolicy.EXCLUDE)
    group_keys, results = gb.aggregate([GroupByRequest(values, [aggregation.sum(), aggregation.mean()])])

`results[i]` is a Table with one column per aggregation of request i, rows
aligned with `group_keys`.  Group order is unspecified, as in libcudf.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import torch

from . import _abi, _lib
from .aggregation import Aggregation
from .column import Column, Table


class TorchAllocator:
    """gbx_allocator over torch's caching allocator (rmm::device_async_resource_ref
    role): scratch and outputs come from torch-owned blocks, freed in stream order."""

    def __init__(self, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.live = {}
        self._alloc_cb = _abi.ALLOC_FN(self._allocate)
        self._dealloc_cb = _abi.DEALLOC_FN(self._deallocate)
        self.struct = _abi.gbx_allocator(None, self._alloc_cb, self._dealloc_cb)
        self.peak = 0
        self.current = 0

    def _allocate(self, ctx, nbytes, stream):
        try:
            t = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        except RuntimeError:
            return None
        p = t.data_ptr()
        self.live[p] = t
        self.current += int(nbytes)
        self.peak = max(self.peak, self.current)
        return p

    def _deallocate(self, ctx, ptr, nbytes, stream):
        t = self.live.pop(ptr, None)
        if t is not None:
            self.current -= int(nbytes)

    def take(self, ptr) -> Optional[torch.Tensor]:
        """Transfers ownership of an allocation to the caller (a result column)."""
        t = self.live.pop(ptr, None)
        if t is not None:
            self.current -= t.numel()
        return t


class GroupByRequest:
    """cudf::groupby::aggregation_request: a value column and its aggregations."""

    def __init__(self, values: Column, aggregations: Sequence[Aggregation]):
        self.values = values
        self.aggregations = list(aggregations)


def _member_column(v: _abi.gbx_column_view, alloc: TorchAllocator) -> Column:
    """A STRUCT result's member (its buffers taken from the allocator)."""
    data = alloc.take(v.data) if v.data else None
    mask = alloc.take(v.null_mask) if v.null_mask else None
    if mask is not None:
        mask = mask.view(torch.int32)
    nc = v.null_count if v.null_count >= 0 else None
    if v.type_id == _abi.TypeId.STRUCT:
        return Column(_abi.TypeId.STRUCT, v.size, None, mask, 0, nc,
                      children=[_member_column(v.dict_keys[i], alloc) for i in range(v.num_children)])
    if v.type_id == _abi.TypeId.STRING:
        ov = v.dict_keys.contents
        offsets = Column(ov.type_id, ov.size, alloc.take(ov.data), None, 0, 0)
        return Column(_abi.TypeId.STRING, v.size, data, mask, 0, nc, dict_keys=offsets)
    return Column(v.type_id, v.size, data, mask, 0, nc, scale=v.scale)


def _result_column(col: _abi.gbx_column, alloc: TorchAllocator, keys_of=None) -> Column:
    v = col.view
    data = alloc.take(col.data) if col.data else None
    mask = alloc.take(col.null_mask) if col.null_mask else None
    if mask is not None:
        mask = mask.view(torch.int32)
    nc = v.null_count if v.null_count >= 0 else None
    if v.type_id == _abi.TypeId.STRUCT:
        return Column(_abi.TypeId.STRUCT, v.size, None, mask, 0, nc,
                      children=[_member_column(v.dict_keys[i], alloc) for i in range(v.num_children)])
    if v.type_id == _abi.TypeId.STRING:
        # the characters, and the offsets child the result also owns
        ov = v.dict_keys.contents
        offs = alloc.take(ov.data)
        offsets = Column(ov.type_id, ov.size, offs, None, 0, 0)
        return Column(_abi.TypeId.STRING, v.size, data, mask, 0, nc, dict_keys=offsets)
    return Column(v.type_id, v.size, data, mask, 0, nc, dict_keys=keys_of,
                  index_type_id=v.index_type_id if v.type_id == _abi.TypeId.DICTIONARY32 else _abi.TypeId.INT32,
                  scale=v.scale)


class GroupBy:
    """cudf::groupby::groupby over the hash path (groupby.hpp:96-199)."""

    def __init__(self, keys: Table, null_handling: _abi.NullPolicy = _abi.NullPolicy.EXCLUDE,
                 keys_are_sorted: _abi.Sorted = _abi.Sorted.NO, column_order=None, null_precedence=None):
        self._keys = keys  # keep the key buffers alive, as pylibcudf does
        self._tv, self._tv_cols = keys.view()
        h = C.c_void_p()
        _lib.check(_lib.lib().gbx_groupby_create(C.byref(self._tv), int(null_handling), int(keys_are_sorted),
                                                 C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().gbx_groupby_destroy(h)
            self._h = None

    def set_strategy(self, strategy: _abi.Strategy) -> None:
        _lib.check(_lib.lib().gbx_groupby_set_strategy(self._h, int(strategy)))

    def set_timing(self, enable: bool = True) -> None:
        """Record per-phase CUDA-event times (see last_stats())."""
        _lib.check(_lib.lib().gbx_groupby_set_timing(self._h, 1 if enable else 0))

    def last_stats(self) -> dict:
        st = _abi.gbx_stats()
        _lib.check(_lib.lib().gbx_groupby_last_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in _abi.gbx_stats._fields_}

    def aggregate(self, requests: List[GroupByRequest], stream: Optional[torch.cuda.Stream] = None,
                  allocator: Optional[TorchAllocator] = None) -> Tuple[Table, List[Table]]:
        """cudf::groupby::groupby::aggregate (groupby.hpp:187-199)."""
        nreq = len(requests)
        reqs = (_abi.gbx_request * max(1, nreq))()
        keep = []
        for i, r in enumerate(requests):
            reqs[i].values = r.values.view()
            keep.append(r.values)
            aggs, kept = _abi.aggregation_array(r.aggregations)
            keep.append(kept)
            reqs[i].num_aggregations = len(r.aggregations)
            reqs[i].aggregations = C.cast(aggs, C.POINTER(_abi.gbx_aggregation))
        st = stream if stream is not None else torch.cuda.current_stream()
        alloc = allocator if allocator is not None else TorchAllocator()
        out = C.POINTER(_abi.gbx_result)()
        with torch.cuda.stream(st):
            status = _lib.lib().gbx_groupby_aggregate(self._h, reqs, nreq, C.c_void_p(st.cuda_stream),
                                                      C.byref(alloc.struct), C.byref(out))
            _lib.check(status)
        try:
            res = out.contents
            key_cols = []
            for c in range(res.num_key_columns):
                kc = self._keys[c]
                key_cols.append(_result_column(res.keys[c], alloc,
                                               keys_of=kc.dict_keys if kc.type_id == _abi.TypeId.DICTIONARY32 else None))
            results = []
            for q in range(res.num_requests):
                ar = res.requests[q]
                results.append(Table([_result_column(ar.results[k], alloc) for k in range(ar.num_results)]))
        finally:
            _lib.lib().gbx_result_release(out)
        return Table(key_cols), results
