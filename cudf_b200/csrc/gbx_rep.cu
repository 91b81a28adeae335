// gbx_rep.cu -- groupby over keys that do not pack into two 64-bit words:
// STRING key columns, or fixed-width columns beyond 128 bits with their null
// bits.
//
// Each row is labelled with the first row inserted of its key -- a table of
// row indices probed by a hash of every key column and resolved by comparing
// the rows' columns themselves, as the reference's set of representative rows
// does for every key (hash/groupby.cu:571-593, row_operators.cuh:1339-1365,
// 1429-1447).  The label is a plain INT32 key, so the groupby proper then runs
// on it with every strategy of the packed-key path; the output keys are the
// original key columns gathered at the representative rows.
//
// Keys the caller declares sorted take the same route with another label:
// the reference's sort path then groups runs of equal adjacent rows in row
// order (sort_helper.cu:96-104, 141-179), or, under EXCLUDE with null keys,
// sorts the rows again (sort_helper.cu:64-71).  Here the label is the run's
// index, or the rank of the key's first row; the groupby runs on it and its
// output is put in label order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_device.cuh"
#include "gbx_kernels.hpp"
#include "gbx_rep.cuh"
#include "gbx_scan.hpp"

namespace gbx {

using namespace dev;

namespace {

// Output column: element g = source element rows[g] (per == 1), or element
// rows[g / per] * per + g % per of a column of `per` elements a group; and
// its validity (null counts added to *nulls).
__global__ void k_gather_fixed(const void* __restrict__ src, int64_t src_offset, const uint32_t* __restrict__ src_mask,
                               int width, int per, const int32_t* __restrict__ rows, int64_t G, void* __restrict__ dst,
                               uint32_t* __restrict__ dst_mask, unsigned long long* nulls)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t g_up   = (G + 31) & ~int64_t(31);
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < g_up; g += stride) {
    bool valid = false;
    if (g < G) {
      const int64_t r = per == 1 ? rows[g] : static_cast<int64_t>(rows[g / per]) * per + g % per;
      valid           = bit_valid(src_mask, r + src_offset);
      const uint64_t v = load_width(src, r + src_offset, width);
      switch (width) {
        case 1: reinterpret_cast<uint8_t*>(dst)[g] = static_cast<uint8_t>(v); break;
        case 2: reinterpret_cast<uint16_t*>(dst)[g] = static_cast<uint16_t>(v); break;
        case 4: reinterpret_cast<uint32_t*>(dst)[g] = static_cast<uint32_t>(v); break;
        default: reinterpret_cast<uint64_t*>(dst)[g] = v; break;
      }
    }
    const uint32_t act = __ballot_sync(0xffffffffu, g < G);
    const uint32_t bal = __ballot_sync(0xffffffffu, g < G && valid);
    if (dst_mask != nullptr && lane == 0 && act) {
      dst_mask[g >> 5] = bal;
      const uint32_t nn = __popc(act & ~bal);
      if (nn) atomicAdd(nulls, static_cast<unsigned long long>(nn));
    }
  }
}

// Validity words of a gathered leaf (its own and its enclosing structs'
// nulls; a negative row is null; null counts added to *nulls).
__global__ void k_gather_leaf_valid(const __grid_constant__ RepCol c, const int32_t* __restrict__ rows, int64_t G,
                                    uint32_t* __restrict__ dst_mask, unsigned long long* nulls)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t g_up   = (G + 31) & ~int64_t(31);
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < g_up; g += stride) {
    const bool valid   = g < G && rows[g] >= 0 && leaf_valid(c, rows[g]);
    const uint32_t act = __ballot_sync(0xffffffffu, g < G);
    const uint32_t bal = __ballot_sync(0xffffffffu, valid);
    if (lane == 0 && act) {
      dst_mask[g >> 5] = bal;
      const uint32_t nn = __popc(act & ~bal);
      if (nn) atomicAdd(nulls, static_cast<unsigned long long>(nn));
    }
  }
}

// STRING output: lengths of the gathered rows (0 for a null row, or a
// negative one).
__global__ void k_gather_str_len(const __grid_constant__ RepCol c, const int32_t* __restrict__ rows, int64_t G,
                                 int64_t* __restrict__ len)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = rows[g];
    int64_t b = 0, l = 0;
    if (r >= 0 && leaf_valid(c, r)) str_span(c, r, b, l);
    len[g] = l;
  }
}

// STRING output: one warp copies each row's characters to its new offset.
__global__ void k_gather_str_copy(const __grid_constant__ RepCol c, const int32_t* __restrict__ rows, int64_t G,
                                  const int64_t* __restrict__ out_offs, unsigned char* __restrict__ out_chars)
{
  const int lane  = threadIdx.x & 31;
  const int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = w; g < G; g += nw) {
    const int64_t r = rows[g];
    if (r < 0 || !leaf_valid(c, r)) continue;
    int64_t b, l;
    str_span(c, r, b, l);
    const auto* s = static_cast<const unsigned char*>(c.data) + b;
    unsigned char* d = out_chars + out_offs[g];
    for (int64_t j = lane; j < l; j += 32) d[j] = s[j];
  }
}

__global__ void k_offsets_out(const int64_t* __restrict__ excl, const int64_t* __restrict__ len, int64_t G,
                              int width, void* __restrict__ out)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g <= G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t v = g < G ? excl[g] : (G > 0 ? excl[G - 1] + len[G - 1] : 0);
    if (width == 4) reinterpret_cast<int32_t*>(out)[g] = static_cast<int32_t>(v);
    else reinterpret_cast<int64_t*>(out)[g] = v;
  }
}



// ---------------------------------------------- MIN / MAX of STRING values

// Lexicographic byte comparison of rows a and b of a STRING leaf (a prefix
// sorts first): <0, 0 or >0, as libcudf compares strings.
__device__ __forceinline__ int str_compare(const RepCol& c, int64_t a, int64_t b)
{
  int64_t ba, la, bb, lb;
  str_span(c, a, ba, la);
  str_span(c, b, bb, lb);
  const auto* s   = static_cast<const unsigned char*>(c.data);
  const int64_t m = la < lb ? la : lb;
  for (int64_t j = 0; j < m; ++j)
    if (s[ba + j] != s[bb + j]) return s[ba + j] < s[bb + j] ? -1 : 1;
  return la < lb ? -1 : (la > lb ? 1 : 0);
}

constexpr int kStrSpin = 1 << 16;

// best[g] = the row of group g's least (greatest) valid string: a row
// replaces the held row by compare-and-swap while its string is strictly
// smaller (greater); bounded (S_SPIN_LIMIT beyond).
__global__ void k_str_extreme(const __grid_constant__ RepCol c, const int32_t* __restrict__ label, int64_t n,
                              bool for_min, int32_t* __restrict__ best, int32_t* status)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t g = label[r];
    if (g < 0 || !leaf_valid(c, r)) continue;
    int32_t cur = best[g];
    int it      = 0;
    for (; it < kStrSpin; ++it) {
      if (cur >= 0) {
        const int cmp = str_compare(c, r, cur);
        if (for_min ? cmp >= 0 : cmp <= 0) break;
      }
      const int32_t old = atomicCAS(best + g, cur, static_cast<int32_t>(r));
      if (old == cur) break;
      cur = old;
    }
    if (it == kStrSpin) atomicOr(status, S_SPIN_LIMIT);
  }
}

// rows[j] = best[labels[j]]: the row whose string each output group takes
// (-1: a group without valid values).
__global__ void k_pick_rows(const int32_t* __restrict__ labels, int64_t G, const int32_t* __restrict__ best,
                            int32_t* __restrict__ rows)
{
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < G;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x)
    rows[j] = best[labels[j]];
}

// ------------------------------------------- keys the caller declares sorted

// start[r] = 1 when row r begins a run: its key differs from row r-1's
// (nulls equal, NaNs equal, sort_helper.cu:141-179).
__global__ void k_run_starts(const __grid_constant__ RepKeys k, int64_t n, uint32_t* __restrict__ start)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    start[r] = (r == 0 || !rep_equal(k, r - 1, r)) ? 1u : 0u;
}

// label[r] = the run of row r (the inclusive scan of the starts, less one);
// first[run] = its first row.
__global__ void k_run_labels(const uint32_t* __restrict__ start, const uint32_t* __restrict__ excl, int64_t n,
                             int32_t* __restrict__ label, int32_t* __restrict__ first)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t id = excl[r] + start[r] - 1u;
    label[r]          = static_cast<int32_t>(id);
    if (start[r]) first[id] = static_cast<int32_t>(r);
  }
}

// fmin[rep] = the smallest row of each representative's key.
__global__ void k_key_first_row(const int32_t* __restrict__ rep, int64_t n, int32_t* __restrict__ fmin)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (rep[r] >= 0) atomicMin(fmin + rep[r], static_cast<int32_t>(r));
}

// mark[r] = 1 when row r is the first row of its key.
__global__ void k_key_first_mark(const int32_t* __restrict__ rep, const int32_t* __restrict__ fmin, int64_t n,
                                 uint32_t* __restrict__ mark)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    mark[r] = (rep[r] >= 0 && fmin[rep[r]] == static_cast<int32_t>(r)) ? 1u : 0u;
}

// label[r] = the rank of the first row of row r's key among the keys' first
// rows (rows with no key keep their label; the mask drops them);
// first[rank] = that row.
__global__ void k_key_labels(const int32_t* __restrict__ rep, const int32_t* __restrict__ fmin,
                             const uint32_t* __restrict__ mark, const uint32_t* __restrict__ excl, int64_t n,
                             int32_t* __restrict__ label, int32_t* __restrict__ first)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (rep[r] < 0) {
      label[r] = 0;
      continue;
    }
    label[r] = static_cast<int32_t>(excl[fmin[rep[r]]]);
    if (mark[r]) first[excl[r]] = static_cast<int32_t>(r);
  }
}

// inv[label of group g] = g: the inner result row of each ordered group.
__global__ void k_order_inverse(const int32_t* __restrict__ labels, int64_t G, int32_t* __restrict__ inv,
                                int32_t* status)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t l = labels[g];
    if (l < 0 || l >= G) {
      atomicOr(status, S_BAD_INDEX);
      continue;
    }
    inv[l] = static_cast<int32_t>(g);
  }
}

// One gathered key column (or struct member): its view and the buffers it
// owns, taken from the result's allocator.
struct Gathered {
  gbx_column_view view{};
  void* data        = nullptr;
  size_t data_bytes = 0;
  uint32_t* mask    = nullptr;
  size_t mask_bytes = 0;
};

struct KeyGather {
  Alloc& a;
  Scratch& sc;
  ResultInternal* internal;
  const KeyTree& t;
  const int32_t* rows;
  int64_t G;
  int num_sms;
  cudaStream_t s;
  bool include;
  unsigned long long* nulls;  // one counter per node
  bool force_mask = false;    // every gathered column gets a mask (rows may be -1)

  // Node `i` gathered at the rows; a key column keeps a mask under INCLUDE
  // only (EXCLUDE dropped its null rows), a struct member whenever it or an
  // enclosing struct may be null (a null struct's members come back null,
  // as a gather of a struct column gives them).
  Gathered node(int i)
  {
    const KeyNode& kn = t.nodes[static_cast<size_t>(i)];
    const RepCol& rc  = t.rk.cols[kn.leaf];
    const gbx_column_view& kv = *kn.v;
    Gathered out;
    out.view.type_id = kv.type_id;
    out.view.scale   = kv.scale;
    out.view.size    = G;
    const bool with_mask =
      force_mask || (rc.top ? (rc.mask != nullptr && include) : (rc.mask != nullptr || rc.nanc > 0));
    if (kv.type_id == GBX_TYPE_STRUCT) {
      internal->arrays.emplace_back();
      auto& members = internal->arrays.back();
      for (int k : kn.kids) {
        Gathered m = node(k);
        if (m.data) internal->extra.emplace_back(m.data, m.data_bytes);
        if (m.mask) internal->extra.emplace_back(m.mask, m.mask_bytes);
        members.push_back(m.view);
      }
      out.view.num_children = static_cast<int32_t>(members.size());
      out.view.dict_keys    = members.data();
    } else if (kv.type_id == GBX_TYPE_STRING) {
      auto* len     = static_cast<int64_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(G, 1)) * 8));
      auto* excl    = static_cast<int64_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(G, 1)) * 8));
      int64_t total = 0;
      if (G > 0) {
        k_gather_str_len<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(rc, rows, G, len);
        GBX_CUDA(cudaGetLastError());
        size_t tb = 0;
        GBX_CUDA(scan_exclusive_i64(nullptr, nullptr, G, nullptr, &tb, s));
        void* temp = sc.get(tb);
        GBX_CUDA(scan_exclusive_i64(len, excl, G, temp, &tb, s));
        int64_t last[2] = {0, 0};
        GBX_CUDA(cudaMemcpyAsync(&last[0], excl + G - 1, 8, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaMemcpyAsync(&last[1], len + G - 1, 8, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaStreamSynchronize(s));
        total = last[0] + last[1];
      }
      const int ow    = total < (int64_t(1) << 31) ? 4 : 8;
      const size_t ob = static_cast<size_t>(G + 1) * ow;
      void* offs_buf  = a.allocate(ob);
      internal->extra.emplace_back(offs_buf, ob);
      out.data_bytes = static_cast<size_t>(std::max<int64_t>(total, 1));
      out.data       = a.allocate(out.data_bytes);
      k_offsets_out<<<grid_of(G + 1, num_sms), kRepBlock, 0, s>>>(excl, len, G, ow, offs_buf);
      GBX_CUDA(cudaGetLastError());
      if (total > 0) {
        k_gather_str_copy<<<grid_of(G * 32, num_sms), kRepBlock, 0, s>>>(rc, rows, G, excl,
                                                                         static_cast<unsigned char*>(out.data));
        GBX_CUDA(cudaGetLastError());
      }
      gbx_column_view ov{};
      ov.type_id = ow == 4 ? GBX_TYPE_INT32 : GBX_TYPE_INT64;
      ov.size    = G + 1;
      ov.data    = offs_buf;
      internal->children.push_back(ov);
      out.view.data      = out.data;
      out.view.dict_keys = &internal->children.back();
    } else {
      int32_t et = kv.type_id;
      if (kv.type_id == GBX_TYPE_DICTIONARY32) {
        et                     = kv.index_type_id ? kv.index_type_id : GBX_TYPE_INT32;
        out.view.index_type_id = et;
        out.view.dict_keys     = kv.dict_keys;
      }
      out.data_bytes = static_cast<size_t>(std::max<int64_t>(G, 1)) * type_width(et);
      out.data       = a.allocate(out.data_bytes);
      out.view.data  = out.data;
      if (G > 0) {
        k_gather_fixed<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(kv.data, rc.offset, nullptr, rc.width, 1, rows, G,
                                                                  out.data, nullptr, nulls + i);
        GBX_CUDA(cudaGetLastError());
      }
    }
    if (with_mask) {
      const size_t words = static_cast<size_t>((G + 31) / 32);
      out.mask_bytes     = std::max<size_t>(((words * 4 + 63) / 64) * 64, 64);
      out.mask           = static_cast<uint32_t*>(a.allocate(out.mask_bytes));
      out.view.null_mask = out.mask;
      out.view.null_count = -1;  // counted below
      if (G > 0) {
        k_gather_leaf_valid<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(rc, rows, G, out.mask, nulls + i);
        GBX_CUDA(cudaGetLastError());
      }
    }
    return out;
  }
};

// Sets the null count of a gathered view and its members from the nodes'
// counters.
void set_null_counts(gbx_column_view& v, const unsigned long long* h, const KeyTree& t, int node)
{
  const KeyNode& kn = t.nodes[static_cast<size_t>(node)];
  if (v.type_id == GBX_TYPE_STRUCT)
    for (size_t m = 0; m < kn.kids.size(); ++m)
      set_null_counts(const_cast<gbx_column_view&>(v.dict_keys[m]), h, t, kn.kids[m]);
  v.null_count = v.null_mask ? static_cast<int64_t>(h[node]) : 0;
}

// A result whose key columns are `keys` gathered at `rows` (G of them, a null
// key kept only under INCLUDE); the caller adds the request columns.
gbx_result* result_with_keys(Alloc& a, Scratch& sc, const std::vector<gbx_column_view>& keys,
                             int32_t null_policy, const KeyTree& t, const int32_t* rows, int64_t G, int num_sms,
                             cudaStream_t s)
{
  const int nkeys = static_cast<int>(keys.size());
  ResultHold hold;
  hold.r    = new gbx_result();
  auto* res = hold.r;
  std::memset(res, 0, sizeof(*res));
  auto* internal       = new ResultInternal{a, {}, {}, {}};
  res->internal        = internal;
  res->num_key_columns = nkeys;
  res->num_groups      = G;
  res->keys            = new gbx_column[nkeys > 0 ? nkeys : 1]();
  const size_t nn      = std::max<size_t>(t.nodes.size(), 1);
  auto* nulls          = static_cast<unsigned long long*>(sc.get(8 * nn));
  GBX_CUDA(cudaMemsetAsync(nulls, 0, 8 * nn, s));
  KeyGather kg{a, sc, internal, t, rows, G, num_sms, s, null_policy == GBX_NULL_INCLUDE, nulls};
  for (int c = 0; c < nkeys; ++c) {
    Gathered g        = kg.node(t.roots[static_cast<size_t>(c)]);
    gbx_column& oc    = res->keys[c];
    oc.view           = g.view;
    oc.data           = g.data;
    oc.data_bytes     = g.data_bytes;
    oc.null_mask      = g.mask;
    oc.mask_bytes     = g.mask_bytes;
  }
  std::vector<unsigned long long> h(nn, 0);
  GBX_CUDA(cudaMemcpyAsync(h.data(), nulls, 8 * nn, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < nkeys; ++c) set_null_counts(res->keys[c].view, h.data(), t, t.roots[static_cast<size_t>(c)]);
  return hold.take();
}

}  // namespace

bool keys_need_representatives(const std::vector<gbx_column_view>& keys, int32_t null_policy)
{
  for (const auto& k : keys)
    if (k.type_id == GBX_TYPE_STRING || k.type_id == GBX_TYPE_STRUCT) return true;
  bool ok = true;
  (void)make_key_plan(keys.data(), static_cast<int>(keys.size()), null_policy,
                      std::vector<int64_t>(keys.size(), -1), ok);
  return !ok;
}

int aggregate_by_representatives(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                                 const gbx_request* requests, int32_t num_requests, void* stream,
                                 const gbx_allocator* mr, gbx_result** out, gbx_stats* stats)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  const int64_t n   = keys.empty() ? 0 : keys[0].size;
  const int num_sms = current_device().num_sms;
  Scratch sc(&a);

  // labels: each row's representative row
  const KeyTree tree = key_tree(keys, null_policy);
  const RepKeys& rk   = tree.rk;
  const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(n) + 2, 64));
  auto* slots  = static_cast<int32_t*>(sc.get(cap * 4));
  auto* rep    = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(n, 1)) * 4));
  auto* status = static_cast<int32_t*>(sc.get(8));
  auto* mask   = static_cast<uint32_t*>(sc.get(static_cast<size_t>((n + 31) / 32) * 4 + 64));
  GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));
  k_fill_i32<<<grid_of(static_cast<int64_t>(cap), num_sms), kRepBlock, 0, s>>>(slots, -1, static_cast<int64_t>(cap));
  GBX_CUDA(cudaGetLastError());
  if (n > 0) {
    k_rep_insert<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rk, n, slots, cap, rep, status);
    GBX_CUDA(cudaGetLastError());
    if (rk.exclude_nulls) {
      k_rep_mask<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, mask);
      GBX_CUDA(cudaGetLastError());
    }
  }
  int32_t h_status = 0;
  GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  if (h_status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "representative table overflow (status 0x%x)", h_status);

  // the groupby on the label
  gbx_column_view label{};
  label.type_id    = GBX_TYPE_INT32;
  label.size       = n;
  label.data       = rep;
  label.null_mask  = rk.exclude_nulls ? mask : nullptr;
  label.null_count = rk.exclude_nulls ? -1 : 0;
  gbx_table_view tv{1, 0, &label};
  gbx_groupby* inner = nullptr;
  ResultHold inner_res;
  int st = gbx_groupby_create(&tv, GBX_NULL_EXCLUDE, 0, &inner);
  if (st == GBX_OK) st = gbx_groupby_set_strategy(inner, groupby_strategy(gb));
  if (st == GBX_OK) st = gbx_groupby_aggregate(inner, requests, num_requests, stream, mr, &inner_res.r);
  if (st == GBX_OK && stats) gbx_groupby_last_stats(inner, stats);
  if (inner) gbx_groupby_destroy(inner);
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
  gbx_result* ir = inner_res.r;

  // the result: the key columns gathered at the labels; the inner result's
  // request columns move over (the same allocator made them)
  const int64_t G  = ir->num_groups;
  const auto* rows = static_cast<const int32_t*>(ir->keys[0].data);
  gbx_result* res  = result_with_keys(a, sc, keys, null_policy, tree, rows, G, num_sms, s);
  res->num_requests = ir->num_requests;
  res->requests     = ir->requests;
  ir->requests      = nullptr;
  ir->num_requests  = 0;
  *out = res;
  return GBX_OK;
}

int aggregate_presorted(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                        const gbx_request* requests, int32_t num_requests, void* stream, const gbx_allocator* mr,
                        gbx_result** out, gbx_stats* stats)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  const int64_t n   = keys.empty() ? 0 : keys[0].size;
  const int num_sms = current_device().num_sms;
  Scratch sc(&a);
  const KeyTree tree = key_tree(keys, null_policy);
  const RepKeys& rk   = tree.rk;
  bool null_keys   = false;
  for (const auto& k : keys) null_keys = null_keys || (k.null_mask != nullptr && k.null_count != 0);
  // EXCLUDE with null keys: the reference sorts the rows again
  // (sort_helper.cu:64-71), so equal keys form one group wherever they sit
  const bool by_key = rk.exclude_nulls && null_keys;

  const size_t nb = static_cast<size_t>(std::max<int64_t>(n, 1)) * 4;
  auto* label     = static_cast<int32_t*>(sc.get(nb));
  auto* first     = static_cast<int32_t*>(sc.get(nb));
  auto* flags     = static_cast<uint32_t*>(sc.get(nb));
  auto* excl      = static_cast<uint32_t*>(sc.get(nb));
  auto* status    = static_cast<int32_t*>(sc.get(8));
  uint32_t* mask  = nullptr;
  GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));
  size_t tb = 0;
  GBX_CUDA(scan_exclusive_u32(nullptr, nullptr, n, nullptr, &tb, s));
  void* temp = sc.get(std::max<size_t>(tb, 1));
  if (!by_key) {
    // runs of equal adjacent rows, in row order
    if (n > 0) {
      k_run_starts<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rk, n, flags);
      GBX_CUDA(cudaGetLastError());
      GBX_CUDA(scan_exclusive_u32(flags, excl, n, temp, &tb, s));
      k_run_labels<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(flags, excl, n, label, first);
      GBX_CUDA(cudaGetLastError());
    }
  } else {
    // one group per key, ordered by the key's first row
    const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(n) + 2, 64));
    auto* slots        = static_cast<int32_t*>(sc.get(cap * 4));
    auto* rep          = static_cast<int32_t*>(sc.get(nb));
    auto* fmin         = static_cast<int32_t*>(sc.get(nb));
    mask               = static_cast<uint32_t*>(sc.get(static_cast<size_t>((n + 31) / 32) * 4 + 64));
    k_fill_i32<<<grid_of(static_cast<int64_t>(cap), num_sms), kRepBlock, 0, s>>>(slots, -1, static_cast<int64_t>(cap));
    GBX_CUDA(cudaGetLastError());
    if (n > 0) {
      k_fill_i32<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(fmin, INT32_MAX, n);
      k_rep_insert<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rk, n, slots, cap, rep, status);
      k_rep_mask<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, mask);
      k_key_first_row<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, fmin);
      k_key_first_mark<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, fmin, n, flags);
      GBX_CUDA(cudaGetLastError());
      GBX_CUDA(scan_exclusive_u32(flags, excl, n, temp, &tb, s));
      k_key_labels<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, fmin, flags, excl, n, label, first);
      GBX_CUDA(cudaGetLastError());
    }
  }
  int32_t h_status = 0;
  GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  if (h_status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "representative table overflow (status 0x%x)", h_status);

  // the groupby on the label: group g of the ordered output has label g
  gbx_column_view lv{};
  lv.type_id    = GBX_TYPE_INT32;
  lv.size       = n;
  lv.data       = label;
  lv.null_mask  = mask;
  lv.null_count = mask ? -1 : 0;
  gbx_table_view tv{1, 0, &lv};
  gbx_groupby* inner = nullptr;
  ResultHold inner_res;
  int st = gbx_groupby_create(&tv, GBX_NULL_EXCLUDE, 0, &inner);
  if (st == GBX_OK) st = gbx_groupby_set_strategy(inner, groupby_strategy(gb));
  if (st == GBX_OK) st = gbx_groupby_aggregate(inner, requests, num_requests, stream, mr, &inner_res.r);
  if (st == GBX_OK && stats) gbx_groupby_last_stats(inner, stats);
  if (inner) gbx_groupby_destroy(inner);
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
  gbx_result* ir = inner_res.r;

  // every request column put in label order
  const int64_t G = ir->num_groups;
  auto* inv       = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(G, 1)) * 4));
  auto* nulls     = static_cast<unsigned long long*>(sc.get(8));
  if (G > 0) {
    k_fill_i32<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(inv, 0, G);
    k_order_inverse<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(static_cast<const int32_t*>(ir->keys[0].data), G, inv,
                                                               status);
    GBX_CUDA(cudaGetLastError());
    GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    if (h_status & S_BAD_INDEX) fail(GBX_ERR_DEVICE, "group label out of range (status 0x%x)", h_status);
  }
  for (int q = 0; q < ir->num_requests && G > 0; ++q)
    for (int k = 0; k < ir->requests[q].num_results; ++k) {
      gbx_column& c = ir->requests[q].results[k];
      const int64_t rows = c.view.size;
      if (rows == 0 || c.data == nullptr) continue;
      GBX_EXPECTS(rows % G == 0, "result column of %lld rows over %lld groups", static_cast<long long>(rows),
                  static_cast<long long>(G));
      const int32_t et = c.view.type_id == GBX_TYPE_DICTIONARY32
                             ? (c.view.index_type_id ? c.view.index_type_id : GBX_TYPE_INT32)
                             : c.view.type_id;
      void* data      = a.allocate(c.data_bytes);
      uint32_t* vmask = c.null_mask ? static_cast<uint32_t*>(a.allocate(c.mask_bytes)) : nullptr;
      k_gather_fixed<<<grid_of(rows, num_sms), kRepBlock, 0, s>>>(c.data, 0, c.null_mask, type_width(et),
                                                                   static_cast<int>(rows / G), inv, rows, data, vmask,
                                                                   nulls);
      GBX_CUDA(cudaGetLastError());
      a.release(c.data, c.data_bytes);
      if (c.null_mask) a.release(c.null_mask, c.mask_bytes);
      c.data      = data;
      c.view.data = data;
      if (c.null_mask) {
        c.null_mask      = vmask;
        c.view.null_mask = vmask;
      }
    }
  // the key columns at each group's first row
  gbx_result* res   = result_with_keys(a, sc, keys, null_policy, tree, first, G, num_sms, s);
  res->num_requests = ir->num_requests;
  res->requests     = ir->requests;
  ir->requests      = nullptr;
  ir->num_requests  = 0;
  *out = res;
  return GBX_OK;
}

bool needs_string_extrema(const gbx_request* requests, int32_t num_requests)
{
  for (int q = 0; q < num_requests; ++q) {
    if (requests[q].values.type_id != GBX_TYPE_STRING) continue;
    for (int k = 0; k < requests[q].num_aggregations; ++k) {
      const int32_t kind = requests[q].aggregations[k].kind;
      if (kind == GBX_AGG_MIN || kind == GBX_AGG_MAX) return true;
    }
  }
  return false;
}

int aggregate_string_extrema(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                             const gbx_request* requests, int32_t num_requests, void* stream,
                             const gbx_allocator* mr, gbx_result** out, gbx_stats* stats)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  const int64_t n   = keys.empty() ? 0 : keys[0].size;
  const int num_sms = current_device().num_sms;
  Scratch sc(&a);
  const size_t n4 = static_cast<size_t>(std::max<int64_t>(n, 1)) * 4;

  // every row's group: the representative row of its key
  const KeyTree tree = key_tree(keys, null_policy);
  const RepKeys& rk  = tree.rk;
  const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(n) + 2, 64));
  auto* slots  = static_cast<int32_t*>(sc.get(cap * 4));
  auto* rep    = static_cast<int32_t*>(sc.get(n4));
  auto* status = static_cast<int32_t*>(sc.get(8));
  auto* mask   = static_cast<uint32_t*>(sc.get(static_cast<size_t>((n + 31) / 32) * 4 + 64));
  GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));
  k_fill_i32<<<grid_of(static_cast<int64_t>(cap), num_sms), kRepBlock, 0, s>>>(slots, -1, static_cast<int64_t>(cap));
  GBX_CUDA(cudaGetLastError());
  if (n > 0) {
    k_rep_insert<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rk, n, slots, cap, rep, status);
    if (rk.exclude_nulls) k_rep_mask<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, mask);
    GBX_CUDA(cudaGetLastError());
  }

  // the requests the groupby on the label answers: every non-STRING
  // request, and the COUNTs of the STRING ones over a stand-in of zeros with
  // their validity; MIN / MAX of the strings each keep a best row per group
  struct Where {
    int q, k;   // original position
    int iq, ik; // position in the inner result (-1: a string extreme)
    int ext;    // index of the string extreme
  };
  struct Extreme {
    RepCol col;
    bool for_min;
    int32_t* best;
  };
  std::vector<Where> where;
  std::vector<Extreme> ext;
  std::vector<gbx_request> reqs;
  std::vector<std::vector<gbx_aggregation>> aggs;
  aggs.reserve(static_cast<size_t>(num_requests) + 1);
  int64_t zbytes = 1;
  for (int q = 0; q < num_requests; ++q)
    if (requests[q].values.type_id == GBX_TYPE_STRING) zbytes = std::max(zbytes, requests[q].values.offset + n);
  void* zeros = sc.get(static_cast<size_t>(zbytes));
  GBX_CUDA(cudaMemsetAsync(zeros, 0, static_cast<size_t>(zbytes), s));
  for (int q = 0; q < num_requests; ++q) {
    const gbx_request& r = requests[q];
    const bool str       = r.values.type_id == GBX_TYPE_STRING;
    int iq               = -1;
    for (int k = 0; k < r.num_aggregations; ++k) {
      const gbx_aggregation& ag = r.aggregations[k];
      if (str && (ag.kind == GBX_AGG_MIN || ag.kind == GBX_AGG_MAX)) {
        const std::vector<gbx_column_view> one{r.values};
        Extreme e{key_tree(one, GBX_NULL_INCLUDE).rk.cols[0], ag.kind == GBX_AGG_MIN,
                  static_cast<int32_t*>(sc.get(n4))};
        where.push_back({q, k, -1, -1, static_cast<int>(ext.size())});
        ext.push_back(e);
        continue;
      }
      if (iq < 0) {
        gbx_request ir = r;
        if (str) {
          gbx_column_view v{};
          v.type_id    = GBX_TYPE_INT8;
          v.size       = r.values.size;
          v.offset     = r.values.offset;
          v.data       = zeros;
          v.null_mask  = r.values.null_mask;
          v.null_count = r.values.null_count;
          ir.values    = v;
        }
        reqs.push_back(ir);
        aggs.emplace_back();
        iq = static_cast<int>(reqs.size()) - 1;
      }
      where.push_back({q, k, iq, static_cast<int>(aggs[iq].size()), -1});
      aggs[iq].push_back(ag);
    }
  }
  if (reqs.empty()) {
    // only string extremes: the groupby still needs one request to run
    gbx_request r{};
    r.values.type_id = GBX_TYPE_INT8;
    r.values.size    = n;
    r.values.data    = zeros;
    reqs.push_back(r);
    aggs.emplace_back(1, gbx_aggregation{});
    aggs.back()[0].kind = GBX_AGG_COUNT_ALL;
  }
  for (size_t i = 0; i < reqs.size(); ++i) {
    reqs[i].num_aggregations = static_cast<int32_t>(aggs[i].size());
    reqs[i].aggregations     = aggs[i].data();
  }
  for (const Extreme& e : ext) {
    k_fill_i32<<<grid_of(std::max<int64_t>(n, 1), num_sms), kRepBlock, 0, s>>>(e.best, -1, std::max<int64_t>(n, 1));
    if (n > 0)
      k_str_extreme<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(e.col, rep, n, e.for_min, e.best, status);
    GBX_CUDA(cudaGetLastError());
  }
  int32_t h_status = 0;
  GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  if (h_status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "representative table overflow (status 0x%x)", h_status);
  if (h_status & S_SPIN_LIMIT) fail(GBX_ERR_DEVICE, "string MIN / MAX update gave up (status 0x%x)", h_status);

  // the groupby on the label
  gbx_column_view lv{};
  lv.type_id    = GBX_TYPE_INT32;
  lv.size       = n;
  lv.data       = rep;
  lv.null_mask  = rk.exclude_nulls ? mask : nullptr;
  lv.null_count = rk.exclude_nulls ? -1 : 0;
  gbx_table_view tv{1, 0, &lv};
  gbx_groupby* inner = nullptr;
  ResultHold inner_res;
  int st = gbx_groupby_create(&tv, GBX_NULL_EXCLUDE, 0, &inner);
  if (st == GBX_OK) st = gbx_groupby_set_strategy(inner, groupby_strategy(gb));
  if (st == GBX_OK)
    st = gbx_groupby_aggregate(inner, reqs.data(), static_cast<int32_t>(reqs.size()), stream, mr, &inner_res.r);
  if (st == GBX_OK && stats) gbx_groupby_last_stats(inner, stats);
  if (inner) gbx_groupby_destroy(inner);
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
  gbx_result* ir = inner_res.r;

  // the result: keys at the labels, the inner columns moved over, each
  // string extreme gathered at its best rows
  const int64_t G     = ir->num_groups;
  const auto* labels  = static_cast<const int32_t*>(ir->keys[0].data);
  ResultHold hold;
  hold.r              = result_with_keys(a, sc, keys, null_policy, tree, labels, G, num_sms, s);
  gbx_result* res     = hold.r;
  auto* internal      = static_cast<ResultInternal*>(res->internal);
  res->num_requests   = num_requests;
  res->requests       = new gbx_aggregation_result[num_requests > 0 ? num_requests : 1]();
  for (int q = 0; q < num_requests; ++q) {
    res->requests[q].num_results = requests[q].num_aggregations;
    res->requests[q].results = new gbx_column[requests[q].num_aggregations > 0 ? requests[q].num_aggregations : 1]();
  }
  auto* rows  = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(G, 1)) * 4));
  auto* nulls = static_cast<unsigned long long*>(sc.get(8));
  for (const Where& w : where) {
    gbx_column& dst = res->requests[w.q].results[w.k];
    if (w.ext < 0) {
      gbx_column& src = ir->requests[w.iq].results[w.ik];
      dst             = src;
      std::memset(&src, 0, sizeof(src));
      continue;
    }
    const Extreme& e = ext[static_cast<size_t>(w.ext)];
    if (G > 0) {
      k_pick_rows<<<grid_of(G, num_sms), kRepBlock, 0, s>>>(labels, G, e.best, rows);
      GBX_CUDA(cudaGetLastError());
    }
    // a one-leaf tree over the value column gathers it like a STRING key,
    // with a mask for the groups that had no valid value (row -1)
    const std::vector<gbx_column_view> one{requests[w.q].values};
    const KeyTree vt = key_tree(one, GBX_NULL_INCLUDE);
    GBX_CUDA(cudaMemsetAsync(nulls, 0, 8, s));
    KeyGather kg{a, sc, internal, vt, rows, G, num_sms, s, true, nulls, true};
    Gathered g = kg.node(vt.roots[0]);
    dst.view       = g.view;
    dst.data       = g.data;
    dst.data_bytes = g.data_bytes;
    dst.null_mask  = g.mask;
    dst.mask_bytes = g.mask_bytes;
    unsigned long long h_nulls = 0;
    GBX_CUDA(cudaMemcpyAsync(&h_nulls, nulls, 8, cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    dst.view.null_count = static_cast<int64_t>(h_nulls);
  }
  GBX_CUDA(cudaStreamSynchronize(s));
  *out = hold.take();
  return GBX_OK;
}

}  // namespace gbx
