"""Served groupby: requests over device-resident columns submitted as they
arrive, run with continuous batching (gbx_server_* in include/gbx.h).

No counterpart in the reference (a libcudf service calls groupby::aggregate
per request from its own threads).

    srv = Server(workers=8, batch_max_rows=200_000)
    t = srv.submit(Table([keys]), [GroupByRequest(values, [aggregation.sum()])])
    group_keys, results, timing = srv.wait(t)

Each result equals ``GroupBy(keys).aggregate(requests)`` on that request
alone.  Result buffers belong to libgbx and are freed when the last tensor
viewing them goes away.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _abi, _lib
from .column import Column, Table
from .groupby import GroupByRequest


class _ResultOwner:
    """Releases a gbx_result once no column views it any more."""

    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        if self.ptr:
            _lib.lib().gbx_result_release(self.ptr)
            self.ptr = None


class _DeviceBytes:
    """A libgbx device allocation seen by torch (no copy)."""

    def __init__(self, ptr: int, nbytes: int, owner: _ResultOwner):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _column(col: _abi.gbx_column, owner: _ResultOwner, device) -> Column:
    v = col.view
    data = torch.as_tensor(_DeviceBytes(col.data, col.data_bytes, owner), device=device) if col.data else None
    mask = None
    if col.null_mask:
        mask = torch.as_tensor(_DeviceBytes(col.null_mask, col.mask_bytes, owner), device=device).view(torch.int32)
    return Column(v.type_id, v.size, data, mask, 0, v.null_count if mask is not None else 0, scale=v.scale)


def request_array(requests: Sequence[GroupByRequest]):
    """gbx_request[] for the C ABI and the host objects it points to."""
    reqs = (_abi.gbx_request * max(1, len(requests)))()
    keep = [reqs]
    for q, r in enumerate(requests):
        reqs[q].values = r.values.view()
        keep.append(r.values)
        aggs, kept = _abi.aggregation_array(r.aggregations)
        keep.append(kept)
        reqs[q].num_aggregations = len(r.aggregations)
        reqs[q].aggregations = C.cast(aggs, C.POINTER(_abi.gbx_aggregation))
    return reqs, keep


class Server:
    """A groupby server on the current CUDA device (gbx_server)."""

    def __init__(self, workers: int = 4, null_handling: _abi.NullPolicy = _abi.NullPolicy.EXCLUDE,
                 hbm_budget_bytes: int = 0, batch_max_rows: int = 0, batch_max_requests: int = 0,
                 large_rows: int = 0, large_in_flight: int = 0):
        self._h = None
        self._held: Dict[int, tuple] = {}
        opts = _abi.gbx_server_options(workers=int(workers), null_policy=int(null_handling),
                                       hbm_budget_bytes=int(hbm_budget_bytes), batch_max_rows=int(batch_max_rows),
                                       batch_max_requests=int(batch_max_requests),
                                       large_in_flight=int(large_in_flight), large_rows=int(large_rows))
        h = C.c_void_p()
        _lib.check(_lib.lib().gbx_server_create(C.byref(opts), C.byref(h)))
        self._h = h
        self._device = torch.device("cuda", torch.cuda.current_device())

    def submit(self, keys: Table, requests: Sequence[GroupByRequest]) -> int:
        tv, cols = keys.view()
        reqs, keep = request_array(requests)
        ticket = C.c_uint64()
        _lib.check(_lib.lib().gbx_server_submit(self._h, C.byref(tv), reqs, len(requests), C.byref(ticket)))
        # the column buffers must live until the request has run
        self._held[ticket.value] = (keys, list(requests))
        return ticket.value

    def wait(self, ticket: int, timeout: Optional[float] = None) -> Tuple[Table, List[Table], dict]:
        out = C.POINTER(_abi.gbx_result)()
        tm = _abi.gbx_server_timing()
        st = _lib.lib().gbx_server_wait(self._h, C.c_uint64(ticket), -1.0 if timeout is None else float(timeout),
                                        C.byref(out), C.byref(tm))
        if st != 0:
            msg = _lib.lib().gbx_last_error() or b""
            if msg.startswith(b"timeout"):
                raise TimeoutError(msg.decode())  # the ticket stays valid
            self._held.pop(ticket, None)
            _lib.check(st)
        self._held.pop(ticket, None)
        timing = {name: getattr(tm, name) for name, _ in _abi.gbx_server_timing._fields_}
        owner = _ResultOwner(out)
        res = out.contents
        keys = Table([_column(res.keys[c], owner, self._device) for c in range(res.num_key_columns)])
        results = []
        for q in range(res.num_requests):
            ar = res.requests[q]
            results.append(Table([_column(ar.results[k], owner, self._device) for k in range(ar.num_results)]))
        return keys, results, timing

    def now(self) -> float:
        return _lib.lib().gbx_server_now(self._h)

    def stats(self) -> dict:
        s = _abi.gbx_server_stats()
        _lib.check(_lib.lib().gbx_server_last_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.gbx_server_stats._fields_}

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().gbx_server_destroy(h)
        self._h = None
        self._held.clear()

    def __del__(self):
        self.close()
