"""GPU test of gbx_groupby_aggregate_noalloc, the groupby for callers that cannot
allocate device memory during the call (an engine that owns the whole GPU
budget through its own pool, or a latency-critical thread on which
cudaMalloc/cudaFree would block).  It must give the same answer as
gbx_groupby_aggregate, call after call, with its scratch in libgbx's fixed
device array and every output buffer passed in by the caller.

Kept in its own file, collected last, so that a run stopping at the first
failure has already run every other test.  Runs alone in a fresh process too.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(n, groups, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(-groups // 2, groups - groups // 2, size=n).astype(np.int64)
    keys[::17] = -1  # the all-ones key word the tables reserve
    a = rng.integers(-1_000_000, 1_000_000, size=n).astype(np.int64)
    b = rng.standard_normal(n).astype(np.float32)
    bvalid = rng.random(n) >= 0.1
    return keys, a, b, bvalid


def _group_scales(keys, x, valid, group_keys):
    """Per-group sum|x|, count and mean x^2 aligned with `group_keys` (the
    error scales of the suite's stated float tolerances)."""
    x = x.astype(np.float64)
    m = np.ones(len(x), bool) if valid is None else valid
    uniq, inv = np.unique(keys, return_inverse=True)
    absx = np.zeros(len(uniq))
    sq = np.zeros(len(uniq))
    cnt = np.zeros(len(uniq))
    np.add.at(absx, inv[m], np.abs(x[m]))
    np.add.at(sq, inv[m], x[m] * x[m])
    np.add.at(cnt, inv[m], 1)
    pos = np.searchsorted(uniq, group_keys)
    return {"abs": absx[pos], "cnt": cnt[pos], "msq": sq[pos] / np.maximum(cnt[pos], 1)}


def _call_noalloc(gb_handle, reqs, nreq, nres, stream, capacity, key_type, result_types):
    """Calls the entry point through the C ABI with caller-owned output buffers."""
    import torch

    from cudf_b200 import _abi, _lib
    from cudf_b200.column import storage_dtype

    words = (capacity + 31) // 32
    keep = []

    def column_buffers(type_id):
        dt = storage_dtype(type_id)
        data = torch.zeros(capacity * dt.itemsize, dtype=torch.uint8, device="cuda")
        mask = torch.zeros(words, dtype=torch.int32, device="cuda")
        keep.extend([data, mask])
        c = _abi.gbx_column()
        c.data = data.data_ptr()
        c.null_mask = mask.data_ptr()
        return c, data, mask

    kc, kdata, kmask = column_buffers(key_type)
    out_keys = (_abi.gbx_column * 1)(kc)
    outs = [column_buffers(t) for t in result_types]
    out_results = (_abi.gbx_column * nres)(*[o[0] for o in outs])
    ng = C.c_int64(-1)
    st = _lib.lib().gbx_groupby_aggregate_noalloc(gb_handle, reqs, nreq, C.c_void_p(stream.cuda_stream),
                                                  out_keys, out_results, capacity, C.byref(ng))
    torch.cuda.synchronize()
    return st, ng.value, out_keys, out_results, (kdata, kmask), [(o[1], o[2]) for o in outs], keep


def _to_numpy(col, data, mask, n):
    from cudf_b200._abi import TypeId
    from cudf_b200.column import storage_dtype, unpack_mask

    dt = storage_dtype(col.view.type_id)
    vals = data.cpu().numpy().view(dt)[:n].copy()
    valid = unpack_mask(mask.cpu().numpy(), n) if col.view.null_mask else None
    return (int(col.view.type_id), vals, valid)


def test_noalloc_matches_aggregate_on_two_calls():
    import torch

    from cudf_b200 import Column, GroupBy, GroupByRequest, Table, _abi, _lib, aggregation as agg
    from cudf_b200._abi import Kind, TypeId
    from tests import gbx_testing as T

    n, groups = 400_000, 20_000
    keys, a, b, bvalid = _inputs(n, groups, seed=2024)
    kcol = Column.from_numpy(keys)
    acol = Column.from_numpy(a)
    bcol = Column.from_numpy(b, bvalid)
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean(), agg.variance()]
    kinds = [x.kind for x in aggs]

    # the existing entry point (gbx_groupby_aggregate, through the Python API)
    gb = GroupBy(Table([kcol]))
    kt, res = gb.aggregate([GroupByRequest(acol, aggs), GroupByRequest(bcol, aggs)])
    want = {"num_groups": kt.num_rows(), "keys": [(int(kt[0].type_id),) + kt[0].to_numpy()],
            "results": [[(int(c.type_id),) + c.to_numpy() for c in t.columns()] for t in res]}

    # the same request through the C ABI, without allocation
    lib = _lib.lib()
    tv, keep_tv = Table([kcol]).view()
    h = C.c_void_p()
    _lib.check(lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)))
    reqs = (_abi.gbx_request * 2)()
    keep = []
    for i, col in enumerate((acol, bcol)):
        reqs[i].values = col.view()
        arr = (_abi.gbx_aggregation * len(aggs))()
        for j, x in enumerate(aggs):
            arr[j].kind = int(x.kind)
            arr[j].ddof = int(x.ddof)
        keep.append(arr)
        reqs[i].num_aggregations = len(aggs)
        reqs[i].aggregations = C.cast(arr, C.POINTER(_abi.gbx_aggregation))
    scales = [_group_scales(keys, a, None, want["keys"][0][1]), _group_scales(keys, b, bvalid, want["keys"][0][1])]
    result_types = [lib.gbx_target_type(int(vt), int(k)) for vt in (TypeId.INT64, TypeId.FLOAT32) for k in kinds]
    stream = torch.cuda.current_stream()
    try:
        for call in range(2):
            st, ng, ok_, or_, kbuf, rbufs, _ = _call_noalloc(h, reqs, 2, len(result_types), stream,
                                                            _abi.NOALLOC_MAX_GROUPS, TypeId.INT64, result_types)
            _lib.check(st)
            assert ng == want["num_groups"], f"call {call}: {ng} groups, expected {want['num_groups']}"
            got = {"num_groups": ng, "keys": [_to_numpy(ok_[0], kbuf[0], kbuf[1], ng)], "results": [[], []]}
            for i in range(len(result_types)):
                got["results"][i // len(aggs)].append(_to_numpy(or_[i], rbufs[i][0], rbufs[i][1], ng))
            go = T.sort_order(got["keys"])
            wo = T.sort_order(want["keys"])
            T.compare_keys(got["keys"], want["keys"], go, wo)
            for q in range(2):
                for k, kind in enumerate(kinds):
                    gcol = got["results"][q][k]
                    wcol = want["results"][q][k]
                    # the same kernels run in both entry points; floating results may
                    # differ only by atomic ordering, bounded by the suite's tolerances
                    scale = var_scale = None
                    if kind == Kind.SUM and q == 1:
                        scale = scales[q]["abs"]
                    elif kind == Kind.MEAN and q == 1:
                        scale = scales[q]["abs"] / np.maximum(scales[q]["cnt"], 1)
                    elif kind == Kind.VARIANCE:
                        var_scale = scales[q]["msq"]
                    T.compare_values(kind, gcol, wcol, go, wo, scale, var_scale, ctx=f"call {call} request {q} {kind.name}")
                    if gcol[2] is not None:
                        assert or_[q * len(aggs) + k].view.null_count == int((~gcol[2]).sum())
    finally:
        lib.gbx_groupby_destroy(h)


def test_noalloc_rejects_too_many_groups():
    import torch

    from cudf_b200 import Column, Table, _abi, _lib
    from cudf_b200._abi import Kind, TypeId

    n = 100_000
    keys = np.arange(n, dtype=np.int64)  # 100k groups > the limit
    kcol = Column.from_numpy(keys)
    vcol = Column.from_numpy(np.ones(n, np.int64))
    lib = _lib.lib()
    tv, keep_tv = Table([kcol]).view()
    h = C.c_void_p()
    _lib.check(lib.gbx_groupby_create(C.byref(tv), 0, 0, C.byref(h)))
    req = (_abi.gbx_request * 1)()
    req[0].values = vcol.view()
    arr = (_abi.gbx_aggregation * 1)()
    arr[0].kind = int(Kind.SUM)
    req[0].num_aggregations = 1
    req[0].aggregations = C.cast(arr, C.POINTER(_abi.gbx_aggregation))
    try:
        st, ng, *_ = _call_noalloc(h, req, 1, 1, torch.cuda.current_stream(), 1024, TypeId.INT64, [TypeId.INT64])
        assert st == _abi.Status.ERR_LOGIC
        assert b"more than 32768 groups" in lib.gbx_last_error()
    finally:
        lib.gbx_groupby_destroy(h)
