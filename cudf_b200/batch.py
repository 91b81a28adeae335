"""Batched hash groupby: many independent groupby instances that share one
schema, aggregated by one CUDA-graph launch (gbx_batch_* in include/gbx.h).

No counterpart in the reference: a libcudf / pylibcudf caller with many
tables loops over ``groupby.GroupBy(keys_i).aggregate(requests_i)``.  Here

    b = BatchGroupBy([BatchInstance(Table([k_i]), [GroupByRequest(v_i, aggs)]) for ...],
                     tune=Tune.MISSING, tune_file="batch_tune.txt")
    res = b.execute()
    keys_i, results_i = res.instance(i)

gives for every instance the same groups and values as ``GroupBy`` on that
instance alone (group order unspecified within an instance).  The input
buffers are read at execute time, so they may be refilled in place between
executes; ``rebind`` points the batch at other buffers of the same shape.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _abi, _lib
from .column import Column, Table
from .groupby import GroupByRequest, TorchAllocator


class BatchInstance:
    """One groupby of a batch: its key table and its requests."""

    def __init__(self, keys: Table, requests: Sequence[GroupByRequest]):
        self.keys = keys
        self.requests = list(requests)


def _instances_array(instances: Sequence[BatchInstance], nreq: int):
    """gbx_batch_instance[] for the C ABI and the host objects it points to."""
    arr = (_abi.gbx_batch_instance * len(instances))()
    keep = []
    for i, inst in enumerate(instances):
        if len(inst.requests) != nreq:
            raise _lib.LogicError(_abi.Status.ERR_LOGIC,
                                  f"batch instance {i} has {len(inst.requests)} requests, instance 0 has {nreq}")
        tv, cols = inst.keys.view()
        keep += [tv, cols]
        arr[i].keys = tv
        reqs = (_abi.gbx_request * max(1, nreq))()
        for q, r in enumerate(inst.requests):
            reqs[q].values = r.values.view()
            keep.append(r.values)
            aggs, kept = _abi.aggregation_array(r.aggregations)
            keep.append(kept)
            reqs[q].num_aggregations = len(r.aggregations)
            reqs[q].aggregations = C.cast(aggs, C.POINTER(_abi.gbx_aggregation))
        keep.append(reqs)
        arr[i].requests = C.cast(reqs, C.POINTER(_abi.gbx_request))
    return arr, keep


class BatchResult:
    """The concatenated groups of every instance (views of the batch's
    output buffers, valid until the next execute / rebind / close)."""

    def __init__(self, offsets: np.ndarray, keys: Table, results: List[Table]):
        self.offsets = offsets
        self.keys = keys
        self.results = results

    @property
    def num_groups(self) -> int:
        return int(self.offsets[-1])

    def instance(self, i: int) -> Tuple[Table, List[Table]]:
        b, e = int(self.offsets[i]), int(self.offsets[i + 1])
        keys = Table([c.slice(b, e) for c in self.keys.columns()])
        results = [Table([c.slice(b, e) for c in t.columns()]) for t in self.results]
        return keys, results


class BatchGroupBy:
    """A batch of groupby instances of one schema (gbx_batch)."""

    def __init__(self, instances: Sequence[BatchInstance],
                 null_handling: _abi.NullPolicy = _abi.NullPolicy.EXCLUDE,
                 tune: _abi.Tune = _abi.Tune.CACHED, tune_file: Optional[str] = None,
                 force_mode: _abi.BatchMode = _abi.BatchMode.AUTO, block_threads: int = 0, tile_rows: int = 0,
                 one_shot: bool = False, stream: Optional[torch.cuda.Stream] = None,
                 allocator: Optional[TorchAllocator] = None):
        self._h = None
        if not instances:
            raise _lib.LogicError(_abi.Status.ERR_LOGIC, "a batch needs at least one instance")
        self._instances = list(instances)
        self._nreq = len(self._instances[0].requests)
        self._alloc = allocator if allocator is not None else TorchAllocator()
        arr, keep = _instances_array(self._instances, self._nreq)
        self._tune_file = tune_file.encode() if tune_file else None
        opts = _abi.gbx_batch_options(null_policy=int(null_handling), tune=int(tune), tune_file=self._tune_file,
                                      force_mode=int(force_mode), block_threads=int(block_threads),
                                      one_shot=1 if one_shot else 0, tile_rows=int(tile_rows))
        st = stream if stream is not None else torch.cuda.current_stream()
        h = C.c_void_p()
        with torch.cuda.stream(st):
            _lib.check(_lib.lib().gbx_batch_create(arr, len(self._instances), self._nreq, C.byref(opts),
                                                   C.c_void_p(st.cuda_stream), C.byref(self._alloc.struct),
                                                   C.byref(h)))
        del keep
        self._h = h

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().gbx_batch_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def num_instances(self) -> int:
        return len(self._instances)

    def rebind(self, instances: Sequence[BatchInstance]) -> None:
        """Reads later executes from these instances' buffers (same schema and row counts)."""
        arr, keep = _instances_array(instances, self._nreq)
        _lib.check(_lib.lib().gbx_batch_rebind(self._h, arr, len(instances)))
        self._instances = list(instances)
        del keep

    def execute(self, stream: Optional[torch.cuda.Stream] = None) -> BatchResult:
        st = stream if stream is not None else torch.cuda.current_stream()
        out = C.POINTER(_abi.gbx_batch_output)()
        _lib.check(_lib.lib().gbx_batch_execute(self._h, C.c_void_p(st.cuda_stream), C.byref(out)))
        o = out.contents
        n = o.num_instances
        offsets = np.ctypeslib.as_array(o.group_offsets, shape=(n + 1,)).copy()
        res = o.columns
        keys = Table([self._column(res.keys[c]) for c in range(res.num_key_columns)])
        results = []
        for q in range(res.num_requests):
            ar = res.requests[q]
            results.append(Table([self._column(ar.results[k]) for k in range(ar.num_results)]))
        return BatchResult(offsets, keys, results)

    def _column(self, col: _abi.gbx_column) -> Column:
        v = col.view
        data = self._alloc.live.get(col.data) if col.data else None
        mask = self._alloc.live.get(col.null_mask) if col.null_mask else None
        if mask is not None:
            mask = mask.view(torch.int32)
        nc = v.null_count if mask is not None else 0
        return Column(v.type_id, v.size, data, mask, 0, nc, scale=v.scale)

    def instance_plan(self) -> dict:
        n = self.num_instances
        modes = np.zeros(n, dtype=np.int32)
        slots = np.zeros(n, dtype=np.int64)
        est = np.zeros(n, dtype=np.int64)
        _lib.check(_lib.lib().gbx_batch_instance_plan(
            self._h, modes.ctypes.data_as(C.POINTER(C.c_int32)), slots.ctypes.data_as(C.POINTER(C.c_int64)),
            est.ctypes.data_as(C.POINTER(C.c_int64))))
        return {"mode": modes, "table_slots": slots, "estimated_groups": est}

    def stats(self) -> dict:
        s = _abi.gbx_batch_stats()
        _lib.check(_lib.lib().gbx_batch_last_stats(self._h, C.byref(s)))
        d = {name: getattr(s, name) for name, _ in _abi.gbx_batch_stats._fields_}
        d["mode_count"] = list(s.mode_count)
        return d
