// gbx_rep.cuh -- keys compared column by column through a representative
// row: the leaves of a key (fixed-width and STRING columns, STRUCT validity),
// their hash and equality, and the table of representative rows.  Shared by
// the groupby over such keys (gbx_rep.cu) and the hash join (gbx_join.cu);
// everything here has internal linkage in each.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_device.cuh"
#include "gbx_host.hpp"

namespace gbx {
namespace {

using namespace dev;

constexpr int kRepBlock  = 256;
constexpr int kKindFixed = 0, kKindF32 = 1, kKindF64 = 2, kKindBool = 3, kKindString = 4, kKindValidity = 5;
// leaves of one key (a STRUCT key is its own validity and its members'
// leaves) and the enclosing structs a leaf inherits nulls from
constexpr int kRepMaxLeaves = 32;
constexpr int kRepMaxDepth  = 4;

// One leaf of the key as the representative table reads it: a fixed-width or
// STRING column, or the validity of a STRUCT column (kKindValidity).
struct RepCol {
  const void* data;      // fixed width: elements; STRING: characters
  const uint32_t* mask;  // own validity (nullptr: all valid)
  int64_t offset;        // element of row 0 (every enclosing struct's offset included)
  const void* offs;      // STRING: offsets (element offset + row)
  int64_t offs_offset;   // STRING: the offsets view's own offset
  int32_t width;         // fixed width: bytes; STRING: bytes of an offset (4 or 8)
  int32_t kind;
  int32_t top;           // a key column itself, not a struct member: EXCLUDE drops rows where it is null
  int32_t nanc;          // enclosing structs with a validity mask
  const uint32_t* anc_mask[kRepMaxDepth];
  int64_t anc_offset[kRepMaxDepth];
};

struct RepKeys {
  int32_t ncols;          // leaves
  int32_t exclude_nulls;  // rows that take no label (any_null)
  int32_t nan_alone;      // distinct rows with NaNs unequal: a row holding a NaN takes no label
  RepCol cols[kRepMaxLeaves];
};

// A leaf is null where it, or a struct enclosing it, is null: a null struct
// row's members read as nulls (the nested comparator compares a struct's
// validity before its members, row_operators.cuh:1456-1500).
__device__ __forceinline__ bool leaf_valid(const RepCol& c, int64_t r)
{
  if (!bit_valid(c.mask, r + c.offset)) return false;
  for (int j = 0; j < c.nanc; ++j)
    if (!bit_valid(c.anc_mask[j], r + c.anc_offset[j])) return false;
  return true;
}

__device__ __forceinline__ uint64_t load_width(const void* p, int64_t i, int w)
{
  switch (w) {
    case 1: return reinterpret_cast<const uint8_t*>(p)[i];
    case 2: return reinterpret_cast<const uint16_t*>(p)[i];
    case 4: return reinterpret_cast<const uint32_t*>(p)[i];
    default: return reinterpret_cast<const uint64_t*>(p)[i];
  }
}

// The value bits that decide equality: -0.0 and +0.0 one value, every NaN one
// value (row_operators.cuh:1285-1312), booleans 0 / 1.
__device__ __forceinline__ uint64_t norm_bits(const RepCol& c, int64_t r)
{
  const int64_t i  = r + c.offset;
  const uint64_t b = load_width(c.data, i, c.width);
  if (c.kind == kKindF32) {
    const float f = __uint_as_float(static_cast<uint32_t>(b));
    if (f != f) return 0x7fc00000u;
    return f == 0.0f ? 0u : b;
  }
  if (c.kind == kKindF64) {
    const double d = __longlong_as_double(static_cast<long long>(b));
    if (d != d) return 0x7ff8000000000000ULL;
    return d == 0.0 ? 0u : b;
  }
  if (c.kind == kKindBool) return b != 0;
  return b;
}

__device__ __forceinline__ void str_span(const RepCol& c, int64_t r, int64_t& begin, int64_t& len)
{
  const int64_t i = r + c.offset + c.offs_offset;
  const int64_t a = static_cast<int64_t>(load_width(c.offs, i, c.width));
  const int64_t b = static_cast<int64_t>(load_width(c.offs, i + 1, c.width));
  begin           = a;
  len             = b - a;
}

// 64-bit hash of a row's key (a null contributes a marker of its own).
__device__ __forceinline__ uint64_t rep_hash(const RepKeys& k, int64_t r)
{
  uint64_t h = 0x2545f4914f6cdd1dULL;
  for (int c = 0; c < k.ncols; ++c) {
    const RepCol& col = k.cols[c];
    uint64_t v;
    if (!leaf_valid(col, r)) {
      v = 0x9e3779b97f4a7c15ULL;
    } else if (col.kind == kKindValidity) {
      v = 1;
    } else if (col.kind == kKindString) {
      int64_t begin, len;
      str_span(col, r, begin, len);
      const auto* s = static_cast<const unsigned char*>(col.data) + begin;
      uint64_t f    = 0xcbf29ce484222325ULL ^ static_cast<uint64_t>(len);  // FNV-1a over the bytes
      for (int64_t j = 0; j < len; ++j) f = (f ^ s[j]) * 0x100000001b3ULL;
      v = f;
    } else {
      v = norm_bits(col, r);
    }
    h = fmix64(h ^ (v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2)));
  }
  return h;
}

// Row a of key `ka` equals row b of key `kb` (two tables whose keys have the
// same leaves): leaf validities equal, and values where valid.
__device__ __forceinline__ bool rep_equal2(const RepKeys& ka, int64_t a, const RepKeys& kb, int64_t b)
{
  for (int c = 0; c < ka.ncols; ++c) {
    const RepCol& ca = ka.cols[c];
    const RepCol& cb = kb.cols[c];
    const bool va    = leaf_valid(ca, a);
    const bool vb    = leaf_valid(cb, b);
    if (va != vb) return false;
    if (!va || ca.kind == kKindValidity) continue;  // nulls are equal (hash/groupby.cu:558)
    if (ca.kind == kKindString) {
      int64_t ba, la, bb, lb;
      str_span(ca, a, ba, la);
      str_span(cb, b, bb, lb);
      if (la != lb) return false;
      const auto* sa = static_cast<const unsigned char*>(ca.data) + ba;
      const auto* sb = static_cast<const unsigned char*>(cb.data) + bb;
      for (int64_t j = 0; j < la; ++j)
        if (sa[j] != sb[j]) return false;
    } else if (norm_bits(ca, a) != norm_bits(cb, b)) {
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ bool rep_equal(const RepKeys& k, int64_t a, int64_t b) { return rep_equal2(k, a, k, b); }

// The row takes no label: exclude_nulls 1 (a groupby under EXCLUDE) drops a
// row with a null key column (the AND of the key columns' own masks,
// hash/groupby.cu:560-567; a null struct member does not count);
// kExcludeAnyNull (a join with nulls unequal) a row with any null leaf,
// which then equals no row (the nested comparator under
// null_equality::UNEQUAL).
constexpr int32_t kExcludeAnyNull = 2;
__device__ __forceinline__ bool any_null(const RepKeys& k, int64_t r)
{
  for (int c = 0; c < k.ncols; ++c) {
    if (k.exclude_nulls == kExcludeAnyNull) {
      if (!leaf_valid(k.cols[c], r)) return true;
    } else if (k.cols[c].top && !bit_valid(k.cols[c].mask, r + k.cols[c].offset)) {
      return true;
    }
  }
  return false;
}

// A valid floating leaf of the row holds a NaN.
__device__ __forceinline__ bool any_nan(const RepKeys& k, int64_t r)
{
  for (int c = 0; c < k.ncols; ++c) {
    const RepCol& col = k.cols[c];
    if ((col.kind != kKindF32 && col.kind != kKindF64) || !leaf_valid(col, r)) continue;
    const uint64_t b = load_width(col.data, r + col.offset, col.width);
    if (col.kind == kKindF32 ? (__uint_as_float(static_cast<uint32_t>(b)) != __uint_as_float(static_cast<uint32_t>(b)))
                             : (__longlong_as_double(static_cast<long long>(b)) !=
                                __longlong_as_double(static_cast<long long>(b))))
      return true;
  }
  return false;
}

// rep[r] = the representative row of row r's key (-1: a null key under
// EXCLUDE); `slots` holds row indices (-1: empty), probed linearly at most
// cap times (S_TABLE_FULL beyond).
__global__ void k_rep_insert(const __grid_constant__ RepKeys k, int64_t n, int32_t* __restrict__ slots, uint64_t cap,
                             int32_t* __restrict__ rep, int32_t* status)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if ((k.exclude_nulls && any_null(k, r)) || (k.nan_alone && any_nan(k, r))) {
      rep[r] = -1;
      continue;
    }
    uint64_t s  = rep_hash(k, r) & (cap - 1);
    int32_t out = -1;
    for (uint64_t p = 0; p < cap; ++p) {
      int32_t cur = slots[s];
      if (cur < 0) {
        const int32_t old = atomicCAS(slots + s, -1, static_cast<int32_t>(r));
        if (old < 0) {
          out = static_cast<int32_t>(r);
          break;
        }
        cur = old;
      }
      if (rep_equal(k, cur, r)) {
        out = cur;
        break;
      }
      s = (s + 1) & (cap - 1);
    }
    if (out < 0) atomicOr(status, S_TABLE_FULL);
    rep[r] = out;
  }
}

// Validity words of the label column: rep >= 0.
__global__ void k_rep_mask(const int32_t* __restrict__ rep, int64_t n, uint32_t* __restrict__ mask)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t n_up   = (n + 31) & ~int64_t(31);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_up; r += stride) {
    const uint32_t bal = __ballot_sync(0xffffffffu, r < n && rep[r] >= 0);
    if (lane == 0) mask[r >> 5] = bal;
  }
}

__global__ void k_fill_i32(int32_t* p, int32_t v, int64_t n)
{
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = v;
}

int grid_of(int64_t n, int num_sms)
{
  const int64_t b = (n + kRepBlock - 1) / kRepBlock;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(num_sms) * 8)));
}

// The key as a tree of columns (STRUCT columns hold their members) and the
// leaves the kernels read.
struct KeyNode {
  const gbx_column_view* v;
  int leaf;               // its leaf (a STRUCT's validity)
  std::vector<int> kids;  // STRUCT: member nodes
};

struct KeyTree {
  RepKeys rk{};
  std::vector<KeyNode> nodes;
  std::vector<int> roots;  // one node per key column
};

int add_key_node(KeyTree& t, const gbx_column_view& v, int64_t base, const RepCol& parent, bool top)
{
  GBX_EXPECTS(t.rk.ncols < kRepMaxLeaves, "a key of more than %d columns and struct members", kRepMaxLeaves);
  const int leaf = t.rk.ncols++;
  RepCol rc{};
  rc.mask   = v.null_count == 0 ? nullptr : v.null_mask;
  rc.offset = base + v.offset;
  rc.data   = v.data;
  rc.top    = top ? 1 : 0;
  rc.nanc   = parent.nanc;
  for (int j = 0; j < parent.nanc; ++j) {
    rc.anc_mask[j]   = parent.anc_mask[j];
    rc.anc_offset[j] = parent.anc_offset[j];
  }
  KeyNode node{&v, leaf, {}};
  if (v.type_id == GBX_TYPE_STRUCT) {
    rc.kind = kKindValidity;
    // members inherit this struct's nulls; their rows start at its offset
    RepCol inherit = rc;
    if (rc.mask != nullptr) {
      GBX_EXPECTS(inherit.nanc < kRepMaxDepth, "struct keys nested deeper than %d levels", kRepMaxDepth);
      inherit.anc_mask[inherit.nanc]   = rc.mask;
      inherit.anc_offset[inherit.nanc] = rc.offset;
      ++inherit.nanc;
    }
    t.rk.cols[leaf] = rc;
    for (int32_t m = 0; m < v.num_children; ++m)
      node.kids.push_back(add_key_node(t, v.dict_keys[m], rc.offset, inherit, false));
  } else if (v.type_id == GBX_TYPE_STRING) {
    rc.kind        = kKindString;
    rc.offs        = v.dict_keys->data;
    rc.offs_offset = v.dict_keys->offset;
    rc.width       = type_width(v.dict_keys->type_id);
    t.rk.cols[leaf] = rc;
  } else {
    const int32_t ty = v.type_id == GBX_TYPE_DICTIONARY32 ? (v.index_type_id ? v.index_type_id : GBX_TYPE_INT32)
                                                          : v.type_id;
    rc.width = type_width(ty);
    rc.kind  = ty == GBX_TYPE_FLOAT32 ? kKindF32 : ty == GBX_TYPE_FLOAT64 ? kKindF64 : ty == GBX_TYPE_BOOL8 ? kKindBool
                                                                                                       : kKindFixed;
    t.rk.cols[leaf] = rc;
  }
  t.nodes.push_back(std::move(node));
  return static_cast<int>(t.nodes.size()) - 1;
}

KeyTree key_tree(const std::vector<gbx_column_view>& keys, int32_t null_policy)
{
  KeyTree t;
  t.rk.exclude_nulls = null_policy == GBX_NULL_EXCLUDE ? 1 : 0;
  const RepCol none{};
  for (const auto& k : keys) t.roots.push_back(add_key_node(t, k, 0, none, true));
  return t;
}

}  // namespace
}  // namespace gbx
