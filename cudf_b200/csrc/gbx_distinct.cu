// gbx_distinct.cu -- distinct rows and a distinct-key hash join on the
// groupby's tables.
//
// distinct_count / distinct_indices (cudf/stream_compaction.hpp:288-424,
// src/stream_compaction/distinct.cu, distinct_count.cu) are the groupby:
// the distinct rows of the keys are its groups, and the row kept per group
// is MIN (KEEP_ANY / KEEP_FIRST) or MAX (KEEP_LAST) of the row index, with
// COUNT_ALL deciding KEEP_NONE -- so every strategy of the groupby (shared
// tables, radix partitions) serves them.  Rows that are distinct on their own
// (a null key under null_equality::UNEQUAL, a NaN key under
// nan_equality::UNEQUAL) are set apart before grouping and appended.
//
// distinct_hash_join (cudf/join.hpp:475-533, src/join/distinct_hash_join.cu):
// the build rows' packed keys go into an open-addressing table with the
// build row of each slot (atomicMin: the first row of a repeated key); every
// probe row then finds its key (no insertion; the probe ends at an empty
// slot) and writes the pair, or for a left join the build row or INT32_MIN.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <limits>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_kernels.hpp"
#include "gbx_table.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kBlock          = 256;
constexpr int32_t kJoinNone   = std::numeric_limits<int32_t>::min();
constexpr uint32_t kNoRowSlot = 0xffffffffu;

int grid_for_rows(int64_t n, int num_sms)
{
  const int64_t b = (n + kBlock - 1) / kBlock;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(num_sms) * 8)));
}

__global__ void k_iota(int32_t* out, int64_t n)
{
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(i);
}

// Whether key column c of row r holds a NaN.
__device__ __forceinline__ bool key_is_nan(const KeyCol& kc, int64_t r)
{
  if (!kc.is_float) return false;
  const int64_t i = r + kc.offset;
  if (kc.width == 4) {
    const float f = reinterpret_cast<const float*>(kc.data)[i];
    return f != f;
  }
  const double d = reinterpret_cast<const double*>(kc.data)[i];
  return d != d;
}

// Rows that are distinct on their own: a null in some key column (when
// nulls_unequal) or a NaN (when nans_unequal) -- NaN of a valid element only.
// `grouped` (a bitmask, may be null) gets 1 for every other row; the rows
// set apart are appended to `alone` (counter *n_alone); `tiebreak` (may be
// null) gets row + 1 for them and 0 otherwise.
__global__ void k_split_alone(const __grid_constant__ KeyPlan kp, int64_t n, bool nulls_unequal, bool nans_unequal,
                              uint32_t* grouped, int32_t* alone, unsigned long long* n_alone, int32_t* tiebreak)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t n_up   = (n + 31) & ~int64_t(31);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_up; r += stride) {
    bool is_alone = false;
    if (r < n) {
      for (int c = 0; c < kp.ncols; ++c) {
        const KeyCol& kc = kp.cols[c];
        const bool valid = bit_valid(kc.mask, r + kc.offset);
        if (!valid && nulls_unequal) is_alone = true;
        if (valid && nans_unequal && key_is_nan(kc, r)) is_alone = true;
      }
    }
    const uint32_t act  = __ballot_sync(0xffffffffu, r < n);
    const uint32_t mine = __ballot_sync(0xffffffffu, r < n && is_alone);
    if (grouped != nullptr && lane == 0 && act) grouped[r >> 5] = act & ~mine;
    if (tiebreak != nullptr && r < n) tiebreak[r] = is_alone ? static_cast<int32_t>(r + 1) : 0;
    if (alone != nullptr && mine) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(n_alone, static_cast<unsigned long long>(__popc(mine)));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (is_alone) alone[base + __popc(mine & ((1u << lane) - 1u))] = static_cast<int32_t>(r);
    } else if (alone == nullptr && mine && lane == 0) {
      atomicAdd(n_alone, static_cast<unsigned long long>(__popc(mine)));
    }
  }
}

// KEEP_NONE: the kept row of every group whose key occurs once.
__global__ void k_select_single(const int32_t* rows, const int32_t* counts, int64_t G, int32_t* out,
                                unsigned long long* n_out)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t g_up   = (G + 31) & ~int64_t(31);
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < g_up; g += stride) {
    const bool keep    = g < G && counts[g] == 1;
    const uint32_t bal = __ballot_sync(0xffffffffu, keep);
    if (bal == 0) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(n_out, static_cast<unsigned long long>(__popc(bal)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) out[base + __popc(bal & ((1u << lane) - 1u))] = rows[g];
  }
}

// ------------------------------------------------------------------ join

// The slot holding key k, or -1: probes until the key or an empty slot
// (at most cap probes); the all-ones key lives in the reserved slot cap.
template <int NW>
__device__ __forceinline__ int64_t find_slot(const TableRef& t, const uint64_t (&k)[NW])
{
  if (key_is_empty<NW>(k)) return *t.special_used ? static_cast<int64_t>(t.cap) : -1;
  const uint64_t mask = t.cap - 1;
  uint64_t s          = hash_key<NW>(k) & mask;
  for (uint64_t p = 0; p < t.cap; ++p) {
    bool hit = true, empty = true;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const uint64_t cur = t.keys[s * NW + w];
      hit                = hit && cur == k[w];
      empty              = empty && cur == kEmptyWord;
    }
    if (hit) return static_cast<int64_t>(s);
    if (empty) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}

template <int NW>
__global__ void k_join_build(const __grid_constant__ KeyPlan kp, const __grid_constant__ TableRef t, int64_t n,
                             uint32_t max_probes, uint32_t* slot_row)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t k[NW];
    if (!pack_key<NW>(kp, r, k)) continue;
    const int64_t s = global_slot<NW>(t, k, max_probes);
    if (s >= 0) atomicMin(slot_row + s, static_cast<uint32_t>(r));
  }
}

// inner: matching (build, probe) pairs appended at *n_out; left: out_build[r]
// for every probe row r.
template <int NW, bool LEFT>
__global__ void k_join_probe(const __grid_constant__ KeyPlan kp, const __grid_constant__ TableRef t, int64_t n,
                             const uint32_t* slot_row, int32_t* out_build, int32_t* out_probe,
                             unsigned long long* n_out)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t n_up   = (n + 31) & ~int64_t(31);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_up; r += stride) {
    int32_t b = kJoinNone;
    if (r < n) {
      uint64_t k[NW];
      if (pack_key<NW>(kp, r, k)) {
        const int64_t s = find_slot<NW>(t, k);
        if (s >= 0 && slot_row[s] != kNoRowSlot) b = static_cast<int32_t>(slot_row[s]);
      }
    }
    if constexpr (LEFT) {
      if (r < n) out_build[r] = b;
    } else {
      const uint32_t bal = __ballot_sync(0xffffffffu, b != kJoinNone);
      if (bal == 0) continue;
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(n_out, static_cast<unsigned long long>(__popc(bal)));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (b != kJoinNone) {
        const unsigned long long at = base + __popc(bal & ((1u << lane) - 1u));
        out_build[at]               = b;
        out_probe[at]               = static_cast<int32_t>(r);
      }
    }
  }
}

__global__ void k_fill_u64_d(uint64_t* p, uint64_t v, int64_t n)
{
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = v;
}

// --------------------------------------------------------------- host side

Alloc make_alloc(const gbx_allocator* mr, cudaStream_t s)
{
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  return a;
}

void check_keys(const gbx_table_view* keys)
{
  GBX_EXPECTS(keys != nullptr && keys->num_columns >= 1 && keys->columns != nullptr, "a key table is needed");
  const int64_t n = keys->columns[0].size;
  for (int c = 0; c < keys->num_columns; ++c) {
    const gbx_column_view& k = keys->columns[c];
    GBX_EXPECTS(k.size == n, "key columns differ in size");
    GBX_EXPECTS(k.size >= 0 && k.offset >= 0, "negative size or offset");
    GBX_EXPECTS(k.size <= INT32_MAX, "row count exceeds cudf::size_type");
    if (k.type_id == GBX_TYPE_DICTIONARY32) GBX_EXPECTS(k.dict_keys != nullptr, "dictionary key column without keys");
    else if (!is_fixed_width(k.type_id))
      fail(GBX_ERR_UNSUPPORTED, "key type %d (string / list / struct / decimal128) is not supported by this library",
           k.type_id);
  }
}

// Packed-key plan of `keys` (INCLUDE: null keys are keys) with every column
// that has a mask treated as nullable; fails beyond 128 bits.
KeyPlan plan_keys(const gbx_table_view* keys, int32_t policy, const std::vector<bool>& nullable)
{
  std::vector<int64_t> key_nulls(keys->num_columns);
  for (int c = 0; c < keys->num_columns; ++c) key_nulls[c] = nullable[c] ? -1 : 0;
  bool ok       = false;
  KeyPlan plan = make_key_plan(keys->columns, keys->num_columns, policy, key_nulls, ok);
  if (!ok) fail(GBX_ERR_UNSUPPORTED, "key columns need more than 128 packed bits; wider composite keys are not supported");
  return plan;
}

// The key columns as k_split_alone reads them (data, mask, offset, width,
// float or not), whatever their packed width.
KeyPlan key_columns(const gbx_table_view* keys)
{
  KeyPlan kp{};
  kp.ncols = keys->num_columns;
  for (int c = 0; c < keys->num_columns; ++c) {
    const gbx_column_view& col = keys->columns[c];
    const int32_t t = col.type_id == GBX_TYPE_DICTIONARY32 ? (col.index_type_id ? col.index_type_id : GBX_TYPE_INT32)
                                                           : col.type_id;
    KeyCol& kc  = kp.cols[c];
    kc.data     = col.data;
    kc.mask     = col.null_mask;
    kc.offset   = col.offset;
    kc.width    = static_cast<int8_t>(type_width(t));
    kc.is_float = is_floating(t) ? 1 : 0;
  }
  return kp;
}

bool any_float_key(const gbx_table_view* keys)
{
  for (int c = 0; c < keys->num_columns; ++c)
    if (is_floating(keys->columns[c].type_id)) return true;
  return false;
}

bool any_mask(const gbx_table_view* keys)
{
  for (int c = 0; c < keys->num_columns; ++c)
    if (keys->columns[c].null_mask != nullptr && keys->columns[c].null_count != 0) return true;
  return false;
}

// RAII of a groupby handle and a result.
struct GroupbyHold {
  gbx_groupby* gb = nullptr;
  gbx_result* res = nullptr;
  ~GroupbyHold()
  {
    if (res) gbx_result_release(res);
    if (gb) gbx_groupby_destroy(gb);
  }
};

void throw_status(int st)
{
  if (st != GBX_OK) fail(st, "%s", g_last_error.c_str());
}

}  // namespace
}  // namespace gbx

using namespace gbx;

extern "C" {

int gbx_distinct_count(const gbx_table_view* keys, int32_t nulls_equal, void* stream, const gbx_allocator* mr,
                       int64_t* out)
{
  return guarded([&] {
    GBX_EXPECTS(out != nullptr, "out is null");
    *out = 0;
    GBX_EXPECTS(nulls_equal == GBX_NULLS_EQUAL || nulls_equal == GBX_NULLS_UNEQUAL, "invalid null_equality");
    if (keys_are_nested_or_strings(keys)) {
      // STRING / STRUCT keys: representative rows (NaNs equal, as here)
      *out = distinct_by_representatives(keys, GBX_KEEP_ANY, nulls_equal, GBX_NANS_EQUAL, stream, mr, nullptr);
      return;
    }
    check_keys(keys);
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    const int64_t n = keys->columns[0].size;
    if (n == 0) return;
    GroupbyHold h;
    const bool unequal = nulls_equal == GBX_NULLS_UNEQUAL && any_mask(keys);
    throw_status(gbx_groupby_create(keys, unequal ? GBX_NULL_EXCLUDE : GBX_NULL_INCLUDE, 0, &h.gb));
    throw_status(gbx_groupby_aggregate(h.gb, nullptr, 0, stream, mr, &h.res));
    int64_t count = h.res->num_groups;
    if (unequal) {
      // every row holding a null is a distinct row of its own
      Alloc a = make_alloc(mr, s);
      Scratch sc(&a);
      const KeyPlan kp = key_columns(keys);
      auto* cnt        = static_cast<unsigned long long*>(sc.get(8));
      GBX_CUDA(cudaMemsetAsync(cnt, 0, 8, s));
      k_split_alone<<<grid_for_rows(n, current_device().num_sms), kBlock, 0, s>>>(kp, n, true, false, nullptr,
                                                                                 nullptr, cnt, nullptr);
      GBX_CUDA(cudaGetLastError());
      unsigned long long h_cnt = 0;
      GBX_CUDA(cudaMemcpyAsync(&h_cnt, cnt, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      count += static_cast<int64_t>(h_cnt);
    }
    *out = count;
  });
}

int gbx_distinct_indices(const gbx_table_view* keys, int32_t keep, int32_t nulls_equal, int32_t nans_equal,
                         void* stream, const gbx_allocator* mr, gbx_column* out)
{
  return guarded([&] {
    GBX_EXPECTS(out != nullptr, "out is null");
    std::memset(out, 0, sizeof(*out));
    GBX_EXPECTS(keep >= GBX_KEEP_ANY && keep <= GBX_KEEP_NONE, "invalid duplicate_keep_option");
    GBX_EXPECTS(nulls_equal == GBX_NULLS_EQUAL || nulls_equal == GBX_NULLS_UNEQUAL, "invalid null_equality");
    GBX_EXPECTS(nans_equal == GBX_NANS_EQUAL || nans_equal == GBX_NANS_UNEQUAL, "invalid nan_equality");
    if (keys_are_nested_or_strings(keys)) {
      // STRING / STRUCT keys: representative rows
      (void)distinct_by_representatives(keys, keep, nulls_equal, nans_equal, stream, mr, out);
      return;
    }
    check_keys(keys);
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    Alloc a         = make_alloc(mr, s);
    const int64_t n = keys->columns[0].size;
    const int nk    = keys->num_columns;
    if (n == 0) {
      alloc_column(a, *out, GBX_TYPE_INT32, 0, 0, false);
      return;
    }
    const int num_sms = current_device().num_sms;
    Scratch sc(&a);

    // rows distinct on their own, and how the rest are grouped:
    //   nulls unequal: a key column 0 whose mask also clears the rows set
    //     apart, grouped under EXCLUDE;
    //   nulls equal, NaNs unequal (float keys): a tie-break key column,
    //     row + 1 on the NaN rows, grouped under INCLUDE
    const bool nulls_apart = nulls_equal == GBX_NULLS_UNEQUAL && any_mask(keys);
    const bool nans_apart  = nans_equal == GBX_NANS_UNEQUAL && any_float_key(keys);
    std::vector<gbx_column_view> cols(keys->columns, keys->columns + nk);
    int32_t policy             = GBX_NULL_INCLUDE;
    int32_t* alone             = nullptr;
    unsigned long long* nalone = nullptr;
    unsigned long long h_alone = 0;
    if (nulls_apart || nans_apart) {
      const KeyPlan kp = key_columns(keys);
      nalone           = static_cast<unsigned long long*>(sc.get(8));
      GBX_CUDA(cudaMemsetAsync(nalone, 0, 8, s));
      if (nulls_apart) {
        auto* grouped = static_cast<uint32_t*>(sc.get(static_cast<size_t>((n + 31) / 32) * 4 + 64));
        alone         = static_cast<int32_t*>(sc.get(static_cast<size_t>(n) * 4));
        k_split_alone<<<grid_for_rows(n, num_sms), kBlock, 0, s>>>(kp, n, true, nans_apart, grouped, alone, nalone,
                                                                   nullptr);
        GBX_CUDA(cudaGetLastError());
        // the grouped rows' mask on column 0, whose view then starts at its
        // first row (the mask is indexed from there)
        const gbx_column_view& c0 = keys->columns[0];
        const int32_t pt0 = c0.type_id == GBX_TYPE_DICTIONARY32 ? (c0.index_type_id ? c0.index_type_id : GBX_TYPE_INT32)
                                                                : c0.type_id;
        cols[0].data       = static_cast<const char*>(c0.data) + c0.offset * type_width(pt0);
        cols[0].offset     = 0;
        cols[0].null_mask  = grouped;
        cols[0].null_count = -1;
        policy             = GBX_NULL_EXCLUDE;
      } else {
        auto* tb = static_cast<int32_t*>(sc.get(static_cast<size_t>(n) * 4));
        k_split_alone<<<grid_for_rows(n, num_sms), kBlock, 0, s>>>(kp, n, false, true, nullptr, nullptr, nalone, tb);
        GBX_CUDA(cudaGetLastError());
        gbx_column_view t{};
        t.type_id    = GBX_TYPE_INT32;
        t.size       = n;
        t.data       = tb;
        t.null_count = 0;
        cols.push_back(t);
        nalone = nullptr;  // the NaN rows are groups of their own here
      }
    }

    // the row kept per group: MIN / MAX of the row index, COUNT_ALL for KEEP_NONE
    auto* iota = static_cast<int32_t*>(sc.get(static_cast<size_t>(n) * 4));
    k_iota<<<grid_for_rows(n, num_sms), kBlock, 0, s>>>(iota, n);
    GBX_CUDA(cudaGetLastError());
    gbx_table_view tv{static_cast<int32_t>(cols.size()), 0, cols.data()};
    gbx_request req{};
    req.values.type_id    = GBX_TYPE_INT32;
    req.values.size       = n;
    req.values.data       = iota;
    req.values.null_count = 0;
    gbx_aggregation aggs[2]{};
    aggs[0].kind         = keep == GBX_KEEP_LAST ? GBX_AGG_MAX : GBX_AGG_MIN;
    aggs[1].kind         = GBX_AGG_COUNT_ALL;
    req.num_aggregations = keep == GBX_KEEP_NONE ? 2 : 1;
    req.aggregations     = aggs;
    GroupbyHold h;
    throw_status(gbx_groupby_create(&tv, policy, 0, &h.gb));
    throw_status(gbx_groupby_aggregate(h.gb, &req, 1, stream, mr, &h.res));
    const int64_t G     = h.res->num_groups;
    const auto* kept    = static_cast<const int32_t*>(h.res->requests[0].results[0].data);
    int64_t n_groups_out = G;
    const int32_t* src   = kept;
    if (keep == GBX_KEEP_NONE && G > 0) {
      auto* single = static_cast<int32_t*>(sc.get(static_cast<size_t>(G) * 4));
      auto* nsel   = static_cast<unsigned long long*>(sc.get(8));
      GBX_CUDA(cudaMemsetAsync(nsel, 0, 8, s));
      k_select_single<<<grid_for_rows(G, num_sms), kBlock, 0, s>>>(
        kept, static_cast<const int32_t*>(h.res->requests[0].results[1].data), G, single, nsel);
      GBX_CUDA(cudaGetLastError());
      unsigned long long h_sel = 0;
      GBX_CUDA(cudaMemcpyAsync(&h_sel, nsel, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      n_groups_out = static_cast<int64_t>(h_sel);
      src          = single;
    }
    if (nalone != nullptr) {
      GBX_CUDA(cudaMemcpyAsync(&h_alone, nalone, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
    }
    const int64_t total = n_groups_out + static_cast<int64_t>(h_alone);
    alloc_column(a, *out, GBX_TYPE_INT32, 0, total, false);
    if (n_groups_out > 0)
      GBX_CUDA(cudaMemcpyAsync(out->data, src, static_cast<size_t>(n_groups_out) * 4, cudaMemcpyDeviceToDevice, s));
    if (h_alone > 0)
      GBX_CUDA(cudaMemcpyAsync(static_cast<int32_t*>(out->data) + n_groups_out, alone, static_cast<size_t>(h_alone) * 4,
                               cudaMemcpyDeviceToDevice, s));
    GBX_CUDA(cudaStreamSynchronize(s));
  });
}

int gbx_distinct_join(const gbx_table_view* build, const gbx_table_view* probe, int32_t compare_nulls,
                      int32_t join_kind, void* stream, const gbx_allocator* mr, gbx_column* build_indices,
                      gbx_column* probe_indices)
{
  return guarded([&] {
    GBX_EXPECTS(build_indices != nullptr && probe_indices != nullptr, "null output");
    std::memset(build_indices, 0, sizeof(*build_indices));
    std::memset(probe_indices, 0, sizeof(*probe_indices));
    check_keys(build);
    check_keys(probe);
    GBX_EXPECTS(build->num_columns == probe->num_columns, "Mismatch in number of columns to be joined on");
    for (int c = 0; c < build->num_columns; ++c) {
      const gbx_column_view &b = build->columns[c], &p = probe->columns[c];
      GBX_EXPECTS(b.type_id == p.type_id && b.scale == p.scale, "Mismatch in joining column data types");
      if (b.type_id == GBX_TYPE_DICTIONARY32)
        fail(GBX_ERR_UNSUPPORTED, "dictionary join keys are not supported by this library");
    }
    GBX_EXPECTS(compare_nulls == GBX_NULLS_EQUAL || compare_nulls == GBX_NULLS_UNEQUAL, "invalid null_equality");
    GBX_EXPECTS(join_kind == 0 || join_kind == 1, "join_kind must be 0 (inner) or 1 (left)");
    cudaStream_t s    = static_cast<cudaStream_t>(stream);
    Alloc a           = make_alloc(mr, s);
    const int64_t nb  = build->columns[0].size;
    const int64_t np  = probe->columns[0].size;
    const int num_sms = current_device().num_sms;
    const int32_t policy = compare_nulls == GBX_NULLS_EQUAL ? GBX_NULL_INCLUDE : GBX_NULL_EXCLUDE;
    // one layout for both sides: a column with a mask on either side is
    // nullable on both
    std::vector<bool> nullable(build->num_columns);
    for (int c = 0; c < build->num_columns; ++c)
      nullable[c] = build->columns[c].null_mask != nullptr || probe->columns[c].null_mask != nullptr;
    const KeyPlan kb = plan_keys(build, policy, nullable);
    const KeyPlan kq = plan_keys(probe, policy, nullable);
    const int NW     = kb.nwords;

    Scratch sc(&a);
    const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(nb) + 2, 64));
    TableRef t{};
    t.cap          = cap;
    t.keys         = static_cast<uint64_t*>(sc.get((cap + 1) * NW * 8));
    t.special_used = static_cast<uint32_t*>(sc.get(8));
    t.status       = static_cast<int32_t*>(sc.get(8));
    auto* slot_row = static_cast<uint32_t*>(sc.get((cap + 1) * 4));
    auto* n_out    = static_cast<unsigned long long*>(sc.get(8));
    k_fill_u64_d<<<grid_for_rows((cap + 1) * NW, num_sms), kBlock, 0, s>>>(t.keys, kEmptyWord, (cap + 1) * NW);
    GBX_CUDA(cudaGetLastError());
    GBX_CUDA(cudaMemsetAsync(slot_row, 0xff, (cap + 1) * 4, s));
    GBX_CUDA(cudaMemsetAsync(t.special_used, 0, 8, s));
    GBX_CUDA(cudaMemsetAsync(t.status, 0, 8, s));
    GBX_CUDA(cudaMemsetAsync(n_out, 0, 8, s));
    const uint32_t max_probes = static_cast<uint32_t>(std::min<uint64_t>(cap, 1u << 12));
    if (nb > 0) {
      if (NW == 1) k_join_build<1><<<grid_for_rows(nb, num_sms), kBlock, 0, s>>>(kb, t, nb, max_probes, slot_row);
      else k_join_build<2><<<grid_for_rows(nb, num_sms), kBlock, 0, s>>>(kb, t, nb, max_probes, slot_row);
      GBX_CUDA(cudaGetLastError());
    }
    if (join_kind == 1) {
      alloc_column(a, *build_indices, GBX_TYPE_INT32, 0, np, false);
      alloc_column(a, *probe_indices, GBX_TYPE_INT32, 0, 0, false);
      if (np > 0) {
        auto* ob = static_cast<int32_t*>(build_indices->data);
        if (NW == 1)
          k_join_probe<1, true><<<grid_for_rows(np, num_sms), kBlock, 0, s>>>(kq, t, np, slot_row, ob, nullptr, n_out);
        else
          k_join_probe<2, true><<<grid_for_rows(np, num_sms), kBlock, 0, s>>>(kq, t, np, slot_row, ob, nullptr, n_out);
        GBX_CUDA(cudaGetLastError());
      }
    } else {
      auto* tb = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(np, 1)) * 4));
      auto* tp = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<int64_t>(np, 1)) * 4));
      if (np > 0) {
        if (NW == 1) k_join_probe<1, false><<<grid_for_rows(np, num_sms), kBlock, 0, s>>>(kq, t, np, slot_row, tb, tp, n_out);
        else k_join_probe<2, false><<<grid_for_rows(np, num_sms), kBlock, 0, s>>>(kq, t, np, slot_row, tb, tp, n_out);
        GBX_CUDA(cudaGetLastError());
      }
      unsigned long long m = 0;
      GBX_CUDA(cudaMemcpyAsync(&m, n_out, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      alloc_column(a, *build_indices, GBX_TYPE_INT32, 0, static_cast<int64_t>(m), false);
      alloc_column(a, *probe_indices, GBX_TYPE_INT32, 0, static_cast<int64_t>(m), false);
      if (m > 0) {
        GBX_CUDA(cudaMemcpyAsync(build_indices->data, tb, m * 4, cudaMemcpyDeviceToDevice, s));
        GBX_CUDA(cudaMemcpyAsync(probe_indices->data, tp, m * 4, cudaMemcpyDeviceToDevice, s));
      }
    }
    int32_t status = 0;
    GBX_CUDA(cudaMemcpyAsync(&status, t.status, 4, cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    if (status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "join table overflow (status 0x%x)", status);
  });
}

void gbx_column_release(gbx_column* col, const gbx_allocator* mr, void* stream)
{
  if (col == nullptr) return;
  Alloc a = make_alloc(mr, static_cast<cudaStream_t>(stream));
  a.release(col->data, col->data_bytes);
  a.release(col->null_mask, col->mask_bytes);
  std::memset(col, 0, sizeof(*col));
}

}  // extern "C"
