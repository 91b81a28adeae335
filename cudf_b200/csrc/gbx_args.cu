// gbx_args.cu -- ARGMIN / ARGMAX of values up to 32 bits as MIN / MAX of a
// packed 64-bit column, so that every strategy computes them.
//
// A 32-bit-or-narrower value's ARGMIN / ARGMAX accumulator is one 64-bit word
// per group -- the value's order key in the high half, the row (ARGMIN) or its
// complement (ARGMAX) in the low half -- kept by a 64-bit min / max (arg_pack,
// gbx_table.cuh).  Only the kernels that read the caller's rows in place know
// each row's index, so a request holding them used to be confined to the
// privatised and global tables.  Here the words are written out as a UINT64
// column first; the request then asks MIN / MAX of it, which the radix
// partitions move like any value, and the group's row is read back from the
// low half (the reference computes ARGMIN / ARGMAX on its hash path,
// hash/groupby.cu:73-84, aggregation.cuh:436-491).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_kernels.hpp"
#include "gbx_table.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kArgBlock = 256;

int grid_of(int64_t n, int num_sms)
{
  const int64_t b = (n + kArgBlock - 1) / kArgBlock;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(num_sms) * 8)));
}

// out[r + ch.offset] = arg_pack(order key, for_min, r) of every valid row.
__global__ void k_arg_words(const __grid_constant__ Channel ch, int64_t n, bool for_min, uint64_t* __restrict__ out,
                            int32_t* status)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t w = 0;
    if (bit_valid(ch.mask, r + ch.offset)) {
      bool ok;
      const uint64_t b = value_bits(ch, r, ok);
      if (!ok) atomicOr(status, S_BAD_INDEX);
      w = arg_pack(arg_order(b, ch.ptype, for_min), for_min, static_cast<uint32_t>(r));
    }
    out[r + ch.offset] = w;
  }
}

// The row of each group from its MIN / MAX word (null groups: -1).
__global__ void k_arg_rows(const uint64_t* __restrict__ w, const uint32_t* __restrict__ mask, int64_t G, bool for_min,
                           int32_t* __restrict__ out)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t lo = static_cast<uint32_t>(w[g]);
    out[g] = bit_valid(mask, g) ? static_cast<int32_t>(for_min ? lo : ~lo) : -1;
  }
}

// The value channel of a column (the fields k_arg_words reads).
Channel value_channel(const gbx_column_view& col)
{
  Channel ch{};
  const int32_t vt = value_type(col);
  ch.data          = col.data;
  ch.mask          = col.null_count == 0 ? nullptr : col.null_mask;
  ch.offset        = col.offset;
  if (col.type_id == GBX_TYPE_DICTIONARY32) {
    const int32_t it = col.index_type_id ? col.index_type_id : GBX_TYPE_INT32;
    ch.dict_data     = col.dict_keys->data;
    ch.dict_offset   = col.dict_keys->offset;
    ch.dict_size     = col.dict_keys->size;
    ch.idx_width     = static_cast<int8_t>(type_width(it));
    ch.idx_signed    = is_unsigned(it) ? 0 : 1;
  }
  ch.ptype    = phys_of(vt);
  ch.is_float = is_floating(vt) ? 1 : 0;
  return ch;
}

}  // namespace

bool args_packable(const gbx_request* requests, int32_t num_requests)
{
  bool any = false;
  for (int q = 0; q < num_requests; ++q)
    for (int k = 0; k < requests[q].num_aggregations; ++k) {
      const int32_t kind = requests[q].aggregations[k].kind;
      if (kind != GBX_AGG_ARGMIN && kind != GBX_AGG_ARGMAX) continue;
      if (type_width(value_type(requests[q].values)) > 4) return false;
      any = true;
    }
  return any;
}

int aggregate_with_packed_args(gbx_groupby* gb, int64_t n, const gbx_request* requests, int32_t num_requests,
                               void* stream, const gbx_allocator* mr, gbx_result** out)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  const int num_sms = current_device().num_sms;
  Scratch sc(&a);
  auto* status = static_cast<int32_t*>(sc.get(8));
  GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));

  // the rewritten requests: each original request without its ARG kinds,
  // then one request per ARG kind over its packed words
  struct Where {
    int q, k;        // original position
    int iq, ik;      // position in the inner result
    bool packed;     // an ARG kind rewritten to MIN / MAX
    bool for_min;
  };
  std::vector<Where> where;
  std::vector<gbx_request> reqs;
  std::vector<std::vector<gbx_aggregation>> aggs;
  aggs.reserve(static_cast<size_t>(num_requests) * 2 + 8);
  for (int q = 0; q < num_requests; ++q) {
    aggs.emplace_back();
    const int iq = static_cast<int>(aggs.size()) - 1;
    gbx_request r = requests[q];
    reqs.push_back(r);
    for (int k = 0; k < requests[q].num_aggregations; ++k) {
      const gbx_aggregation& ag = requests[q].aggregations[k];
      if (ag.kind == GBX_AGG_ARGMIN || ag.kind == GBX_AGG_ARGMAX) continue;
      where.push_back({q, k, iq, static_cast<int>(aggs[iq].size()), false, false});
      aggs[iq].push_back(ag);
    }
  }
  for (int q = 0; q < num_requests; ++q) {
    for (int k = 0; k < requests[q].num_aggregations; ++k) {
      const gbx_aggregation& ag = requests[q].aggregations[k];
      if (ag.kind != GBX_AGG_ARGMIN && ag.kind != GBX_AGG_ARGMAX) continue;
      const bool for_min = ag.kind == GBX_AGG_ARGMIN;
      const gbx_column_view& v = requests[q].values;
      const Channel ch         = value_channel(v);
      auto* words = static_cast<uint64_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(n + v.offset, 1)) * 8));
      if (n > 0) {
        k_arg_words<<<grid_of(n, num_sms), kArgBlock, 0, s>>>(ch, n, for_min, words, status);
        GBX_CUDA(cudaGetLastError());
      }
      gbx_request r{};
      r.values.type_id    = GBX_TYPE_UINT64;
      r.values.size       = n;
      r.values.offset     = v.offset;
      r.values.data       = words;
      r.values.null_mask  = ch.mask;
      r.values.null_count = ch.mask ? v.null_count : 0;
      aggs.emplace_back(1, gbx_aggregation{});
      aggs.back()[0].kind = for_min ? GBX_AGG_MIN : GBX_AGG_MAX;
      reqs.push_back(r);
      where.push_back({q, k, static_cast<int>(aggs.size()) - 1, 0, true, for_min});
    }
  }
  for (size_t i = 0; i < reqs.size(); ++i) {
    reqs[i].num_aggregations = static_cast<int32_t>(aggs[i].size());
    reqs[i].aggregations     = aggs[i].data();
  }
  int32_t h_status = 0;
  GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  if (h_status & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");

  // the groupby with the rewritten requests (no ARG kind left)
  ResultHold inner_res;
  const int st = gbx_groupby_aggregate(gb, reqs.data(), static_cast<int32_t>(reqs.size()), stream, mr, &inner_res.r);
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
  gbx_result* ir = inner_res.r;

  // the result in the caller's request order
  ResultHold out_res;
  out_res.r = new gbx_result();
  auto* res = out_res.r;
  std::memset(res, 0, sizeof(*res));
  res->internal        = ir->internal;  // the same allocator made every column
  ir->internal         = nullptr;
  res->num_key_columns = ir->num_key_columns;
  res->keys            = ir->keys;
  ir->keys             = nullptr;
  ir->num_key_columns  = 0;
  res->num_groups      = ir->num_groups;
  res->num_requests    = num_requests;
  res->requests        = new gbx_aggregation_result[num_requests > 0 ? num_requests : 1]();
  for (int q = 0; q < num_requests; ++q) {
    res->requests[q].num_results = requests[q].num_aggregations;
    res->requests[q].results = new gbx_column[requests[q].num_aggregations > 0 ? requests[q].num_aggregations : 1]();
  }
  const int64_t G = ir->num_groups;
  for (const Where& w : where) {
    gbx_column& src = ir->requests[w.iq].results[w.ik];
    gbx_column& dst = res->requests[w.q].results[w.k];
    if (!w.packed) {
      dst = src;
    } else {
      // INT32 rows from the words; the validity is the MIN / MAX result's
      alloc_column(a, dst, GBX_TYPE_INT32, 0, G, false);
      if (G > 0) {
        k_arg_rows<<<grid_of(G, num_sms), kArgBlock, 0, s>>>(static_cast<const uint64_t*>(src.data), src.null_mask, G,
                                                              w.for_min, static_cast<int32_t*>(dst.data));
        GBX_CUDA(cudaGetLastError());
      }
      dst.null_mask       = src.null_mask;
      dst.mask_bytes      = src.mask_bytes;
      dst.view.null_mask  = src.null_mask;
      dst.view.null_count = src.view.null_count;
      a.release(src.data, src.data_bytes);
    }
    std::memset(&src, 0, sizeof(src));
  }
  GBX_CUDA(cudaStreamSynchronize(s));
  *out = out_res.take();
  return GBX_OK;
}

bool needs_count_stand_ins(const gbx_request* requests, int32_t num_requests)
{
  for (int q = 0; q < num_requests; ++q)
    if (counted_only(requests[q].values.type_id)) return true;
  return false;
}

// COUNT_VALID / COUNT_ALL over a column the kernels do not read (STRING,
// LIST, STRUCT, DECIMAL128): only its rows' validity matters, so the request
// runs over an INT8 column of zeros with the same offset, size and mask.
int aggregate_with_count_stand_ins(gbx_groupby* gb, int64_t n, const gbx_request* requests, int32_t num_requests,
                                   void* stream, const gbx_allocator* mr, gbx_result** out)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  int64_t bytes = 1;
  for (int q = 0; q < num_requests; ++q)
    if (counted_only(requests[q].values.type_id)) bytes = std::max(bytes, requests[q].values.offset + n);
  Scratch sc(&a);
  void* zeros = sc.get(static_cast<size_t>(bytes));
  GBX_CUDA(cudaMemsetAsync(zeros, 0, static_cast<size_t>(bytes), s));
  std::vector<gbx_request> reqs(requests, requests + num_requests);
  for (gbx_request& r : reqs) {
    if (!counted_only(r.values.type_id)) continue;
    gbx_column_view v{};
    v.type_id    = GBX_TYPE_INT8;
    v.size       = r.values.size;
    v.offset     = r.values.offset;
    v.data       = zeros;
    v.null_mask  = r.values.null_mask;
    v.null_count = r.values.null_count;
    r.values     = v;
  }
  const int st = gbx_groupby_aggregate(gb, reqs.data(), num_requests, stream, mr, out);
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
  // the stand-in's release is stream-ordered after the call's kernels
  return GBX_OK;
}

}  // namespace gbx
