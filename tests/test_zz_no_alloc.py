"""GPU tests of gbx_groupby_aggregate_noalloc, the groupby for callers that
cannot allocate device memory during the call: an engine whose own pool owns
the whole GPU budget, or a latency-critical thread on which cudaMalloc /
cudaFree would block or synchronise the device.

Each case calls the entry point through the C ABI twice in a row, with every
output buffer passed in by the caller, and checks both results against the
oracle (keys, COUNT and integer results bit-exact after a sort by key, floats
within the suite's stated bounds).  It also checks the property the entry
point exists for: across a call made after the set-up call, the device's free
memory, torch's reserved memory and the default stream-ordered pool's
reserved and used bytes do not change.

Kept in its own file, collected last, so that a run stopping at the first
failure has already run every other test.  Runs alone in a fresh process too.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cudf_b200._abi import Kind, NullPolicy, TypeId
from oracle.oracle import HostCol
from tests import gbx_testing as T

pytestmark = pytest.mark.gpu

ALL6 = [(Kind.SUM, 0), (Kind.COUNT_VALID, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1)]


def _device_memory():
    """Free device bytes, torch's reserved bytes, and the default pool's
    reserved and used bytes on device 0."""
    import torch
    from cuda.bindings import runtime as rt

    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info(0)
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    attrs = []
    for a in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent):
        err, v = rt.cudaMemPoolGetAttribute(pool, a)
        assert err == rt.cudaError_t.cudaSuccess
        attrs.append(int(v))
    return {"free": int(free), "torch_reserved": int(torch.cuda.memory_reserved(0)),
            "pool_reserved": attrs[0], "pool_used": attrs[1]}


class NoAllocCall:
    """One groupby object over device key columns and requests, called through
    gbx_groupby_aggregate_noalloc with caller-owned outputs."""

    def __init__(self, key_cols, requests, null_policy):
        from cudf_b200 import Table, _abi, _lib

        self.lib = _lib.lib()
        self._abi = _abi
        self.key_cols = key_cols
        self.tv, self._keep_tv = Table(key_cols).view()
        self.h = C.c_void_p()
        _lib.check(self.lib.gbx_groupby_create(C.byref(self.tv), int(null_policy), 0, C.byref(self.h)))
        self.reqs = (_abi.gbx_request * len(requests))()
        self._keep = []
        self.result_types = []
        for i, (col, aggs) in enumerate(requests):
            self.reqs[i].values = col.view()
            arr, kept = _abi.aggregation_array(aggs)
            self._keep.append(kept)
            self.reqs[i].num_aggregations = len(aggs)
            self.reqs[i].aggregations = C.cast(arr, C.POINTER(_abi.gbx_aggregation))
            vt = col.dict_keys.type_id if col.type_id == TypeId.DICTIONARY32 else col.type_id
            self.result_types += [self.lib.gbx_target_type(int(vt), int(a[0])) for a in aggs]
        self.aggs_per_req = [len(a) for _, a in requests]

    def outputs(self, capacity):
        """Caller-owned output buffers: keys at their own width (a dictionary
        key at its index width), results at their target type's."""
        import torch

        from cudf_b200.column import storage_dtype

        words = (capacity + 31) // 32 + 16
        bufs = []

        def column(type_id):
            dt = storage_dtype(type_id)
            data = torch.zeros(max(capacity, 1) * dt.itemsize, dtype=torch.uint8, device="cuda")
            mask = torch.zeros(words, dtype=torch.int32, device="cuda")
            c = self._abi.gbx_column()
            c.data = data.data_ptr()
            c.null_mask = mask.data_ptr()
            bufs.append((data, mask))
            return c

        ktypes = [k.index_type_id if k.type_id == TypeId.DICTIONARY32 else k.type_id for k in self.key_cols]
        out_keys = (self._abi.gbx_column * len(ktypes))(*[column(t) for t in ktypes])
        out_results = (self._abi.gbx_column * len(self.result_types))(*[column(t) for t in self.result_types])
        return {"capacity": capacity, "keys": out_keys, "results": out_results, "bufs": bufs}

    def call(self, out, stream=None):
        import torch

        stream = stream or torch.cuda.current_stream()
        ng = C.c_int64(-1)
        st = self.lib.gbx_groupby_aggregate_noalloc(self.h, self.reqs, len(self.aggs_per_req),
                                                    C.c_void_p(stream.cuda_stream), out["keys"], out["results"],
                                                    out["capacity"], C.byref(ng))
        torch.cuda.synchronize()
        return st, ng.value

    def to_host(self, out, ng):
        """The call's outputs in the oracle's result structure."""
        from cudf_b200.column import storage_dtype, unpack_mask

        def col(c, data, mask):
            tid = c.view.type_id
            dt = storage_dtype(c.view.index_type_id if tid == TypeId.DICTIONARY32 else tid)
            vals = data.cpu().numpy().view(dt)[:ng].copy()
            if tid == TypeId.BOOL8:
                vals = vals.astype(bool)
            valid = unpack_mask(mask.cpu().numpy(), ng) if c.view.null_mask else None
            if valid is not None:
                assert c.view.null_count == int((~valid).sum()), "reported null count differs from the mask"
            return (int(tid), vals, valid)

        nk = len(out["keys"])
        got = {"num_groups": ng, "keys": [col(out["keys"][i], *out["bufs"][i]) for i in range(nk)], "results": []}
        o = 0
        for n in self.aggs_per_req:
            got["results"].append([col(out["results"][o + j], *out["bufs"][nk + o + j]) for j in range(n)])
            o += n
        return got

    def close(self):
        self.lib.gbx_groupby_destroy(self.h)


def _two_calls_against_oracle(host_keys, host_reqs, key_cols, dev_reqs, policy, capacity):
    """Set-up call on an empty slice, then two calls in a row, each checked
    against the oracle; the second is bracketed by memory readings."""
    from cudf_b200 import _lib

    # zero rows: the set-up call (loads the scratch array and the kernels)
    empty = NoAllocCall([k.slice(0, 0) for k in key_cols], [(c.slice(0, 0), a) for c, a in dev_reqs], policy)
    try:
        out0 = empty.outputs(16)
        st, ng = empty.call(out0)
        _lib.check(st)
        assert ng == 0
    finally:
        empty.close()

    nc = NoAllocCall(key_cols, dev_reqs, policy)
    try:
        for call in range(2):
            out = nc.outputs(capacity)
            before = _device_memory()
            st, ng = nc.call(out)
            after = _device_memory()
            _lib.check(st)
            assert after == before, f"call {call} changed device memory: {before} -> {after}"
            got = nc.to_host(out, ng)
            T.assert_parity(host_keys, host_reqs, policy, gpu=got)
    finally:
        nc.close()


def test_noalloc_matches_oracle_on_two_calls():
    from cudf_b200 import Column

    rng = np.random.default_rng(2024)
    n, groups = 400_000, 20_000
    keys = rng.integers(-groups // 2, groups - groups // 2, size=n).astype(np.int64)
    keys[::17] = -1  # the all-ones key word the tables reserve
    a = rng.integers(-1_000_000, 1_000_000, size=n).astype(np.int64)
    b = rng.standard_normal(n).astype(np.float32)
    bvalid = rng.random(n) >= 0.1
    host_keys = [HostCol(keys)]
    host_reqs = [(HostCol(a), ALL6), (HostCol(b, bvalid), ALL6)]
    key_cols = [Column.from_numpy(keys)]
    dev_reqs = [(Column.from_numpy(a), ALL6), (Column.from_numpy(b, bvalid), ALL6)]
    _two_calls_against_oracle(host_keys, host_reqs, key_cols, dev_reqs, NullPolicy.EXCLUDE, 32_768)


def test_noalloc_nullable_keys_include():
    """Two nullable key columns under INCLUDE: null keys form groups, and the
    output keys carry validity masks filled by the call."""
    from cudf_b200 import Column

    rng = np.random.default_rng(77)
    n = 300_000
    k1 = rng.integers(0, 60, size=n).astype(np.int32)
    k2 = rng.integers(-40, 40, size=n).astype(np.int16)
    v1 = rng.random(n) >= 0.05
    v2 = rng.random(n) >= 0.08
    x = 1e6 + rng.standard_normal(n)
    aggs = [(Kind.SUM, 0), (Kind.MEAN, 0), (Kind.VARIANCE, 1), (Kind.COUNT_ALL, 0), (Kind.MAX, 0)]
    host_keys = [HostCol(k1, v1), HostCol(k2, v2)]
    key_cols = [Column.from_numpy(k1, v1), Column.from_numpy(k2, v2)]
    _two_calls_against_oracle(host_keys, [(HostCol(x), aggs)], key_cols, [(Column.from_numpy(x), aggs)],
                              NullPolicy.INCLUDE, 8_192)


def test_noalloc_dictionary_key_with_int64_indices():
    """A DICTIONARY32 key with 64-bit indices: its output holds the indices,
    8 bytes per row, into the input's dictionary."""
    from cudf_b200 import Column

    rng = np.random.default_rng(91)
    n = 250_000
    dict_vals = rng.permutation(np.arange(-500, 500, dtype=np.int64) * 7919)
    idx = rng.integers(0, len(dict_vals), size=n).astype(np.int64)
    valid = rng.random(n) >= 0.03
    v = rng.integers(-1_000, 1_000, size=n).astype(np.int32)
    aggs = [(Kind.SUM, 0), (Kind.MIN, 0), (Kind.MAX, 0), (Kind.COUNT_VALID, 0), (Kind.MEAN, 0)]
    host_keys = [HostCol(idx, valid, dict_keys=HostCol(dict_vals))]
    kcol = Column.dictionary(Column.from_numpy(idx, valid), Column.from_numpy(dict_vals))
    _two_calls_against_oracle(host_keys, [(HostCol(v), aggs)], [kcol], [(Column.from_numpy(v), aggs)],
                              NullPolicy.EXCLUDE, 2_048)


def test_noalloc_rejects_too_many_groups():
    from cudf_b200 import Column

    n = 100_000
    keys = np.arange(n, dtype=np.int64)  # 100k groups > the limit
    nc = NoAllocCall([Column.from_numpy(keys)], [(Column.from_numpy(np.ones(n, np.int64)), [(Kind.SUM, 0)])],
                     NullPolicy.EXCLUDE)
    try:
        st, ng = nc.call(nc.outputs(1024))
        assert st == nc._abi.Status.ERR_LOGIC
        assert b"more than 32768 groups" in nc.lib.gbx_last_error()
    finally:
        nc.close()
