// gbx_join.cu -- hash joins with repeated keys: inner, left, full, left semi
// and left anti (cudf::inner_join / left_join / full_join, join.hpp:107-190,
// join/join.cu:33-118; left_semi_join / left_anti_join, join.hpp:200-260,
// join/semi_join.cu).
//
// The reference builds a multimap from each build row's hash to its row and
// probes it twice (once to size the output, once to write it), comparing
// rows on every hash hit (join/hash_join.cu:150-330).  Here the build rows are
// grouped by key first: a table of representative rows (gbx_rep.cuh; full
// key comparison on collisions, so any key type the representative path
// takes -- fixed-width, STRING, STRUCT) gives each build row its key's
// representative, a count per representative and a scan place the build rows
// of each key next to each other.  A probe row then finds its key's
// representative once, reads the key's row count (the output size is an
// exclusive scan of those counts) and copies the key's rows out: the probe
// compares keys once per probe row, not once per build row of its key.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_rep.cuh"
#include "gbx_scan.hpp"

namespace gbx {

using namespace dev;

namespace {

constexpr int32_t kJoinNoneValue = INT32_MIN;  // cudf::JoinNoneValue (join.hpp)

// rows of each build key: cnt[rep]++ for every labelled build row
__global__ void k_key_counts(const int32_t* __restrict__ rep, int64_t n, uint32_t* __restrict__ cnt)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (rep[r] >= 0) atomicAdd(cnt + rep[r], 1u);
}

// The build rows of each key at start[rep] + [0, cnt[rep]) of `rows`.
__global__ void k_key_place(const int32_t* __restrict__ rep, int64_t n, const uint32_t* __restrict__ start,
                            uint32_t* __restrict__ fill, int32_t* __restrict__ rows)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t k = rep[r];
    if (k < 0) continue;
    rows[start[k] + atomicAdd(fill + k, 1u)] = static_cast<int32_t>(r);
  }
}

// Each probe row's build representative (-1: none) and its output rows:
// the key's build rows (inner), at least one (left, full), one if it has a
// match (semi) or one if it has none (anti).
__global__ void k_probe_find(const __grid_constant__ RepKeys kb, const __grid_constant__ RepKeys kp, int64_t n,
                             const int32_t* __restrict__ slots, uint64_t cap, const uint32_t* __restrict__ cnt,
                             int32_t kind, int32_t* __restrict__ match, int64_t* __restrict__ nout)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t found = -1;
    if (!(kp.exclude_nulls && any_null(kp, r))) {
      uint64_t s = rep_hash(kp, r) & (cap - 1);
      for (uint64_t p = 0; p < cap; ++p) {
        const int32_t cur = slots[s];
        if (cur < 0) break;
        if (rep_equal2(kb, cur, kp, r)) {
          found = cur;
          break;
        }
        s = (s + 1) & (cap - 1);
      }
    }
    const int64_t c = found >= 0 ? cnt[found] : 0;
    int64_t o;
    switch (kind) {
      case GBX_JOIN_INNER: o = c; break;
      case GBX_JOIN_LEFT_SEMI: o = c > 0 ? 1 : 0; break;
      case GBX_JOIN_LEFT_ANTI: o = c > 0 ? 0 : 1; break;
      default: o = c > 0 ? c : 1; break;  // left, full
    }
    match[r] = found;
    nout[r]  = o;
  }
}

// The (probe, build) index pairs of every probe row from its first output
// row `at`; semi / anti write the probe row alone.  Full joins mark the
// matched keys.
__global__ void k_probe_emit(const int32_t* __restrict__ match, const int64_t* __restrict__ nout,
                             const int64_t* __restrict__ at, int64_t n, const uint32_t* __restrict__ start,
                             const int32_t* __restrict__ rows, int32_t kind, int32_t* __restrict__ out_probe,
                             int32_t* __restrict__ out_build, uint8_t* __restrict__ matched)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t o = nout[r];
    if (o == 0) continue;
    const int64_t b = at[r];
    if (kind == GBX_JOIN_LEFT_SEMI || kind == GBX_JOIN_LEFT_ANTI) {
      out_probe[b] = static_cast<int32_t>(r);
      continue;
    }
    const int32_t k = match[r];
    if (k < 0) {
      out_probe[b] = static_cast<int32_t>(r);
      out_build[b] = kJoinNoneValue;
      continue;
    }
    if (matched != nullptr) matched[k] = 1;
    const uint32_t first = start[k];
    for (int64_t j = 0; j < o; ++j) {
      out_probe[b + j] = static_cast<int32_t>(r);
      out_build[b + j] = rows[first + j];
    }
  }
}

// Full join: build rows whose key no probe row matched (or that took no
// label), flagged for the compaction.
__global__ void k_build_unmatched(const int32_t* __restrict__ rep, int64_t n, const uint8_t* __restrict__ matched,
                                  uint32_t* __restrict__ flag)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    flag[r] = (rep[r] < 0 || matched[rep[r]] == 0) ? 1u : 0u;
}

__global__ void k_append_unmatched(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, int64_t n,
                                   uint64_t base, int32_t* __restrict__ out_probe, int32_t* __restrict__ out_build)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (!flag[r]) continue;
    out_probe[base + pos[r]] = kJoinNoneValue;
    out_build[base + pos[r]] = static_cast<int32_t>(r);
  }
}

// ------------------------------------------------- distinct rows, any keys

// Per key (indexed by its representative row): first and last row, rows.
__global__ void k_rep_stats(const int32_t* __restrict__ rep, int64_t n, int32_t* __restrict__ fmin,
                            int32_t* __restrict__ fmax, uint32_t* __restrict__ cnt)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t k = rep[r];
    if (k < 0) continue;
    atomicMin(fmin + k, static_cast<int32_t>(r));
    atomicMax(fmax + k, static_cast<int32_t>(r));
    atomicAdd(cnt + k, 1u);
  }
}

// flag[r] = 1 when row r is kept: a row distinct on its own (no label), or
// its key's row by the keep option (KEEP_ANY: the representative).
__global__ void k_rep_keep(const int32_t* __restrict__ rep, int64_t n, const int32_t* __restrict__ fmin,
                           const int32_t* __restrict__ fmax, const uint32_t* __restrict__ cnt, int32_t keep,
                           uint32_t* __restrict__ flag)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t k = rep[r];
    bool kept;
    if (k < 0) kept = true;
    else if (keep == GBX_KEEP_FIRST) kept = fmin[k] == r;
    else if (keep == GBX_KEEP_LAST) kept = fmax[k] == r;
    else if (keep == GBX_KEEP_NONE) kept = k == r && cnt[k] == 1;
    else kept = k == r;
    flag[r] = kept ? 1u : 0u;
  }
}

__global__ void k_compact_rows(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, int64_t n,
                               int32_t* __restrict__ out)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (flag[r]) out[pos[r]] = static_cast<int32_t>(r);
}

// Both key tables must have the same columns: type, scale and, for STRUCT
// columns, the same members.
void check_join_keys(const gbx_column_view& a, const gbx_column_view& b)
{
  GBX_EXPECTS(a.type_id == b.type_id && a.scale == b.scale, "Mismatch in joining column data types");
  if (a.type_id == GBX_TYPE_DICTIONARY32)
    fail(GBX_ERR_UNSUPPORTED, "dictionary join keys are not supported by this library");
  if (a.type_id == GBX_TYPE_STRUCT) {
    GBX_EXPECTS(a.num_children == b.num_children && a.dict_keys != nullptr && b.dict_keys != nullptr &&
                  a.num_children > 0,
                "Mismatch in joining column data types");
    for (int32_t m = 0; m < a.num_children; ++m) {
      GBX_EXPECTS(a.dict_keys[m].size >= a.offset + a.size && b.dict_keys[m].size >= b.offset + b.size,
                  "a struct member is shorter than its struct");
      check_join_keys(a.dict_keys[m], b.dict_keys[m]);
    }
  } else if (a.type_id == GBX_TYPE_STRING) {
    for (const gbx_column_view* v : {&a, &b}) {
      GBX_EXPECTS(v->dict_keys != nullptr && (v->dict_keys->type_id == GBX_TYPE_INT32 ||
                                              v->dict_keys->type_id == GBX_TYPE_INT64),
                  "a STRING key column needs its INT32 / INT64 offsets column");
      GBX_EXPECTS(v->size == 0 || v->dict_keys->size >= v->offset + v->size + 1, "offsets column too short");
    }
  } else if (!is_fixed_width(a.type_id)) {
    fail(GBX_ERR_UNSUPPORTED, "join key type %d (list / decimal128) is not supported by this library", a.type_id);
  }
}

void check_table(const gbx_table_view* t)
{
  GBX_EXPECTS(t != nullptr && t->num_columns >= 1 && t->columns != nullptr, "a key table is needed");
  for (int c = 0; c < t->num_columns; ++c) {
    GBX_EXPECTS(t->columns[c].size == t->columns[0].size, "key columns differ in size");
    GBX_EXPECTS(t->columns[c].size >= 0 && t->columns[c].offset >= 0, "negative size or offset");
    GBX_EXPECTS(t->columns[c].size <= INT32_MAX, "row count exceeds cudf::size_type");
  }
}

}  // namespace

bool keys_are_nested_or_strings(const gbx_table_view* keys)
{
  if (keys == nullptr || keys->columns == nullptr) return false;
  for (int c = 0; c < keys->num_columns; ++c)
    if (keys->columns[c].type_id == GBX_TYPE_STRING || keys->columns[c].type_id == GBX_TYPE_STRUCT) return true;
  return false;
}

int64_t distinct_by_representatives(const gbx_table_view* keys, int32_t keep, int32_t nulls_equal,
                                    int32_t nans_equal, void* stream, const gbx_allocator* mr, gbx_column* out)
{
  check_table(keys);
  for (int c = 0; c < keys->num_columns; ++c) check_join_keys(keys->columns[c], keys->columns[c]);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Alloc a;
  a.st = s;
  if (mr && mr->allocate && mr->deallocate) {
    a.user     = *mr;
    a.has_user = true;
  }
  const int64_t n = keys->columns[0].size;
  if (n == 0) {
    if (out) alloc_column(a, *out, GBX_TYPE_INT32, 0, 0, false);
    return 0;
  }
  const int num_sms = current_device().num_sms;
  const std::vector<gbx_column_view> cols(keys->columns, keys->columns + keys->num_columns);
  KeyTree t          = key_tree(cols, GBX_NULL_INCLUDE);
  t.rk.exclude_nulls = nulls_equal == GBX_NULLS_UNEQUAL ? kExcludeAnyNull : 0;
  t.rk.nan_alone     = nans_equal == GBX_NANS_UNEQUAL ? 1 : 0;

  Scratch sc(&a);
  const size_t n4    = static_cast<size_t>(n) * 4;
  const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(n) + 2, 64));
  auto* slots  = static_cast<int32_t*>(sc.get(cap * 4));
  auto* rep    = static_cast<int32_t*>(sc.get(n4));
  auto* fmin   = static_cast<int32_t*>(sc.get(n4));
  auto* fmax   = static_cast<int32_t*>(sc.get(n4));
  auto* cnt    = static_cast<uint32_t*>(sc.get(n4));
  auto* flag   = static_cast<uint32_t*>(sc.get(n4));
  auto* pos    = static_cast<uint32_t*>(sc.get(n4));
  auto* status = static_cast<int32_t*>(sc.get(8));
  GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));
  GBX_CUDA(cudaMemsetAsync(cnt, 0, n4, s));
  k_fill_i32<<<grid_of(static_cast<int64_t>(cap), num_sms), kRepBlock, 0, s>>>(slots, -1, static_cast<int64_t>(cap));
  k_fill_i32<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(fmin, INT32_MAX, n);
  k_fill_i32<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(fmax, -1, n);
  k_rep_insert<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(t.rk, n, slots, cap, rep, status);
  k_rep_stats<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, fmin, fmax, cnt);
  k_rep_keep<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(rep, n, fmin, fmax, cnt, keep, flag);
  GBX_CUDA(cudaGetLastError());
  size_t tb = 0;
  GBX_CUDA(scan_exclusive_u32(nullptr, nullptr, n, nullptr, &tb, s));
  void* temp = sc.get(std::max<size_t>(tb, 1));
  GBX_CUDA(scan_exclusive_u32(flag, pos, n, temp, &tb, s));
  uint32_t last[2] = {0, 0};
  int32_t h_status = 0;
  GBX_CUDA(cudaMemcpyAsync(&last[0], pos + n - 1, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaMemcpyAsync(&last[1], flag + n - 1, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
  GBX_CUDA(cudaStreamSynchronize(s));
  if (h_status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "representative table overflow (status 0x%x)", h_status);
  const int64_t kept = static_cast<int64_t>(last[0]) + last[1];
  if (out) {
    alloc_column(a, *out, GBX_TYPE_INT32, 0, kept, false);
    if (kept > 0) {
      k_compact_rows<<<grid_of(n, num_sms), kRepBlock, 0, s>>>(flag, pos, n, static_cast<int32_t*>(out->data));
      GBX_CUDA(cudaGetLastError());
    }
    GBX_CUDA(cudaStreamSynchronize(s));
  }
  return kept;
}

}  // namespace gbx

using namespace gbx;

extern "C" {

int gbx_hash_join(const gbx_table_view* left, const gbx_table_view* right, int32_t compare_nulls, int32_t join_kind,
                  void* stream, const gbx_allocator* mr, gbx_column* left_indices, gbx_column* right_indices)
{
  return guarded([&] {
    GBX_EXPECTS(left_indices != nullptr && right_indices != nullptr, "null output");
    std::memset(left_indices, 0, sizeof(*left_indices));
    std::memset(right_indices, 0, sizeof(*right_indices));
    check_table(left);
    check_table(right);
    GBX_EXPECTS(left->num_columns == right->num_columns, "Mismatch in number of columns to be joined on");
    for (int c = 0; c < left->num_columns; ++c) check_join_keys(left->columns[c], right->columns[c]);
    GBX_EXPECTS(compare_nulls == GBX_NULLS_EQUAL || compare_nulls == GBX_NULLS_UNEQUAL, "invalid null_equality");
    GBX_EXPECTS(join_kind >= GBX_JOIN_INNER && join_kind <= GBX_JOIN_LEFT_ANTI, "invalid join kind %d", join_kind);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Alloc a;
    a.st = s;
    if (mr && mr->allocate && mr->deallocate) {
      a.user     = *mr;
      a.has_user = true;
    }
    const int num_sms = current_device().num_sms;

    // build the smaller side of an inner join (join.cu:53-63), else the right
    const bool swap = join_kind == GBX_JOIN_INNER && right->columns[0].size > left->columns[0].size;
    const gbx_table_view* build = swap ? left : right;
    const gbx_table_view* probe = swap ? right : left;
    const int64_t nb = build->columns[0].size;
    const int64_t np = probe->columns[0].size;
    const std::vector<gbx_column_view> bcols(build->columns, build->columns + build->num_columns);
    const std::vector<gbx_column_view> pcols(probe->columns, probe->columns + probe->num_columns);
    KeyTree tb = key_tree(bcols, GBX_NULL_INCLUDE);
    KeyTree tp = key_tree(pcols, GBX_NULL_INCLUDE);
    const int32_t excl      = compare_nulls == GBX_NULLS_UNEQUAL ? kExcludeAnyNull : 0;
    tb.rk.exclude_nulls     = excl;
    tp.rk.exclude_nulls     = excl;
    const RepKeys& kb       = tb.rk;
    const RepKeys& kp       = tp.rk;

    Scratch sc(&a);
    const size_t nb4 = static_cast<size_t>(std::max<int64_t>(nb, 1)) * 4;
    const size_t np4 = static_cast<size_t>(std::max<int64_t>(np, 1)) * 4;
    const uint64_t cap = next_pow2(std::max<uint64_t>(2 * static_cast<uint64_t>(nb) + 2, 64));
    auto* slots  = static_cast<int32_t*>(sc.get(cap * 4));
    auto* rep    = static_cast<int32_t*>(sc.get(nb4));
    auto* cnt    = static_cast<uint32_t*>(sc.get(nb4));
    auto* start  = static_cast<uint32_t*>(sc.get(nb4));
    auto* fill   = static_cast<uint32_t*>(sc.get(nb4));
    auto* rows   = static_cast<int32_t*>(sc.get(nb4));
    auto* match  = static_cast<int32_t*>(sc.get(np4));
    auto* nout   = static_cast<int64_t*>(sc.get(np4 * 2));
    auto* at     = static_cast<int64_t*>(sc.get(np4 * 2));
    auto* status = static_cast<int32_t*>(sc.get(8));
    GBX_CUDA(cudaMemsetAsync(status, 0, 8, s));
    GBX_CUDA(cudaMemsetAsync(cnt, 0, nb4, s));
    GBX_CUDA(cudaMemsetAsync(fill, 0, nb4, s));
    k_fill_i32<<<grid_of(static_cast<int64_t>(cap), num_sms), kRepBlock, 0, s>>>(slots, -1, static_cast<int64_t>(cap));
    GBX_CUDA(cudaGetLastError());
    size_t tb32 = 0, tb64 = 0;
    GBX_CUDA(scan_exclusive_u32(nullptr, nullptr, std::max<int64_t>(nb, 1), nullptr, &tb32, s));
    GBX_CUDA(scan_exclusive_i64(nullptr, nullptr, std::max<int64_t>(np, 1), nullptr, &tb64, s));
    size_t tbytes = std::max(tb32, tb64);
    void* temp    = sc.get(std::max<size_t>(tbytes, 1));

    // 1. the build rows grouped by key
    if (nb > 0) {
      k_rep_insert<<<grid_of(nb, num_sms), kRepBlock, 0, s>>>(kb, nb, slots, cap, rep, status);
      k_key_counts<<<grid_of(nb, num_sms), kRepBlock, 0, s>>>(rep, nb, cnt);
      GBX_CUDA(cudaGetLastError());
      GBX_CUDA(scan_exclusive_u32(cnt, start, nb, temp, &tbytes, s));
      k_key_place<<<grid_of(nb, num_sms), kRepBlock, 0, s>>>(rep, nb, start, fill, rows);
      GBX_CUDA(cudaGetLastError());
    }
    // 2. each probe row's key and output rows, their first output row
    uint64_t total = 0;
    if (np > 0) {
      k_probe_find<<<grid_of(np, num_sms), kRepBlock, 0, s>>>(kb, kp, np, slots, cap, cnt, join_kind, match, nout);
      GBX_CUDA(cudaGetLastError());
      GBX_CUDA(scan_exclusive_i64(nout, at, np, temp, &tbytes, s));
      int64_t last[2] = {0, 0};
      GBX_CUDA(cudaMemcpyAsync(&last[0], at + np - 1, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaMemcpyAsync(&last[1], nout + np - 1, 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      total = static_cast<uint64_t>(last[0] + last[1]);
    }
    int32_t h_status = 0;
    GBX_CUDA(cudaMemcpyAsync(&h_status, status, 4, cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    if (h_status & S_TABLE_FULL) fail(GBX_ERR_DEVICE, "join table overflow (status 0x%x)", h_status);
    GBX_EXPECTS(total <= static_cast<uint64_t>(INT32_MAX), "the join's output exceeds cudf::size_type rows");

    // 3. full joins: the build rows no probe row matched
    const bool full       = join_kind == GBX_JOIN_FULL;
    uint8_t* matched      = nullptr;
    uint32_t* flag        = nullptr;
    uint32_t* pos         = nullptr;
    uint64_t n_unmatched  = 0;
    if (full) {
      matched = static_cast<uint8_t*>(sc.get(std::max<int64_t>(nb, 1)));
      GBX_CUDA(cudaMemsetAsync(matched, 0, std::max<int64_t>(nb, 1), s));
    }
    const bool pairs = join_kind != GBX_JOIN_LEFT_SEMI && join_kind != GBX_JOIN_LEFT_ANTI;
    gbx_column& out_probe = swap ? *right_indices : *left_indices;
    gbx_column& out_build = swap ? *left_indices : *right_indices;
    // the output size of a full join is known once the matches are marked
    int32_t* probe_buf = nullptr;
    int32_t* build_buf = nullptr;
    if (!full) {
      alloc_column(a, out_probe, GBX_TYPE_INT32, 0, static_cast<int64_t>(total), false);
      alloc_column(a, out_build, GBX_TYPE_INT32, 0, pairs ? static_cast<int64_t>(total) : 0, false);
      probe_buf = static_cast<int32_t*>(out_probe.data);
      build_buf = static_cast<int32_t*>(out_build.data);
    } else {
      probe_buf = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<uint64_t>(total, 1)) * 4));
      build_buf = static_cast<int32_t*>(sc.get(static_cast<size_t>(std::max<uint64_t>(total, 1)) * 4));
    }
    if (np > 0 && total > 0) {
      k_probe_emit<<<grid_of(np, num_sms), kRepBlock, 0, s>>>(match, nout, at, np, start, rows, join_kind, probe_buf,
                                                              build_buf, matched);
      GBX_CUDA(cudaGetLastError());
    }
    if (full) {
      if (nb > 0) {
        flag = static_cast<uint32_t*>(sc.get(nb4));
        pos  = static_cast<uint32_t*>(sc.get(nb4));
        k_build_unmatched<<<grid_of(nb, num_sms), kRepBlock, 0, s>>>(rep, nb, matched, flag);
        GBX_CUDA(cudaGetLastError());
        GBX_CUDA(scan_exclusive_u32(flag, pos, nb, temp, &tbytes, s));
        uint32_t last[2] = {0, 0};
        GBX_CUDA(cudaMemcpyAsync(&last[0], pos + nb - 1, 4, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaMemcpyAsync(&last[1], flag + nb - 1, 4, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaStreamSynchronize(s));
        n_unmatched = static_cast<uint64_t>(last[0]) + last[1];
      }
      const int64_t m = static_cast<int64_t>(total + n_unmatched);
      alloc_column(a, out_probe, GBX_TYPE_INT32, 0, m, false);
      alloc_column(a, out_build, GBX_TYPE_INT32, 0, m, false);
      if (total > 0) {
        GBX_CUDA(cudaMemcpyAsync(out_probe.data, probe_buf, total * 4, cudaMemcpyDeviceToDevice, s));
        GBX_CUDA(cudaMemcpyAsync(out_build.data, build_buf, total * 4, cudaMemcpyDeviceToDevice, s));
      }
      if (n_unmatched > 0) {
        k_append_unmatched<<<grid_of(nb, num_sms), kRepBlock, 0, s>>>(flag, pos, nb, total,
                                                                      static_cast<int32_t*>(out_probe.data),
                                                                      static_cast<int32_t*>(out_build.data));
        GBX_CUDA(cudaGetLastError());
      }
    }
    GBX_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
