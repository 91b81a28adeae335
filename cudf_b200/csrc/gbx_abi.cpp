// gbx_abi.cpp -- host side of libgbx: the C ABI (include/gbx.h) over the
// sm_100a kernels.  Restates the reference's host flow of
// cudf::groupby::groupby::aggregate (cpp/src/groupby/groupby.cu:150-221) and
// detail::hash::groupby (cpp/src/groupby/hash/groupby.cu:548-667):
// validation, empty-input shortcut, flattening of compound aggregations,
// table build + single-pass aggregation, compaction and finalisation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_kernels.hpp"
#include "gbx_sort.hpp"

namespace gbx {

thread_local std::string g_last_error;

[[noreturn]] void fail(int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Failure{code, buf};
}

// ------------------------------------------------------------------- types

int type_width(int32_t t)
{
  switch (t) {
    case GBX_TYPE_INT8:
    case GBX_TYPE_UINT8:
    case GBX_TYPE_BOOL8: return 1;
    case GBX_TYPE_INT16:
    case GBX_TYPE_UINT16: return 2;
    case GBX_TYPE_INT32:
    case GBX_TYPE_UINT32:
    case GBX_TYPE_FLOAT32:
    case GBX_TYPE_TIMESTAMP_DAYS:
    case GBX_TYPE_DURATION_DAYS:
    case GBX_TYPE_DECIMAL32: return 4;
    case GBX_TYPE_INT64:
    case GBX_TYPE_UINT64:
    case GBX_TYPE_FLOAT64:
    case GBX_TYPE_TIMESTAMP_SECONDS:
    case GBX_TYPE_TIMESTAMP_MILLISECONDS:
    case GBX_TYPE_TIMESTAMP_MICROSECONDS:
    case GBX_TYPE_TIMESTAMP_NANOSECONDS:
    case GBX_TYPE_DURATION_SECONDS:
    case GBX_TYPE_DURATION_MILLISECONDS:
    case GBX_TYPE_DURATION_MICROSECONDS:
    case GBX_TYPE_DURATION_NANOSECONDS:
    case GBX_TYPE_DECIMAL64: return 8;
    default: return 0;
  }
}

bool is_integral(int32_t t) { return (t >= GBX_TYPE_INT8 && t <= GBX_TYPE_UINT64) || t == GBX_TYPE_BOOL8; }
bool is_floating(int32_t t) { return t == GBX_TYPE_FLOAT32 || t == GBX_TYPE_FLOAT64; }
bool is_duration(int32_t t) { return t >= GBX_TYPE_DURATION_DAYS && t <= GBX_TYPE_DURATION_NANOSECONDS; }
bool is_decimal(int32_t t) { return t == GBX_TYPE_DECIMAL32 || t == GBX_TYPE_DECIMAL64; }
bool is_fixed_width(int32_t t) { return type_width(t) > 0; }
bool is_unsigned(int32_t t) { return t >= GBX_TYPE_UINT8 && t <= GBX_TYPE_UINT64; }

// Physical code of a fixed-width element type.
int8_t phys_of(int32_t t)
{
  if (t == GBX_TYPE_BOOL8) return P_BOOL;
  if (t == GBX_TYPE_FLOAT32) return P_F32;
  if (t == GBX_TYPE_FLOAT64) return P_F64;
  int w = type_width(t);
  if (is_unsigned(t)) return w == 1 ? P_U8 : w == 2 ? P_U16 : w == 4 ? P_U32 : P_U64;
  return w == 1 ? P_I8 : w == 2 ? P_I16 : w == 4 ? P_I32 : P_I64;
}

// cudf::detail::target_type restated (detail/aggregation/aggregation.hpp:1212-1335)
// for the kinds the hash path computes (hash/groupby.cu:73-84); GBX_TYPE_EMPTY
// when the combination is invalid.
int32_t target_type(int32_t t, int32_t kind)
{
  if (!is_fixed_width(t)) return GBX_TYPE_EMPTY;
  switch (kind) {
    case GBX_AGG_SUM:
      if (is_integral(t)) return GBX_TYPE_INT64;
      if (is_floating(t) || is_duration(t) || is_decimal(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_PRODUCT:
    case GBX_AGG_SUM_OF_SQUARES:
      if (is_integral(t)) return GBX_TYPE_INT64;
      if (is_floating(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_MIN:
    case GBX_AGG_MAX: return t;
    case GBX_AGG_ARGMIN:
    case GBX_AGG_ARGMAX: return GBX_TYPE_INT32;  // size_type row index
    case GBX_AGG_COUNT_VALID:
    case GBX_AGG_COUNT_ALL: return GBX_TYPE_INT32;
    case GBX_AGG_MEAN:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      if (is_duration(t) || is_decimal(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_VARIANCE:
    case GBX_AGG_STD:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      return GBX_TYPE_EMPTY;
    // the sort-path kinds (detail/aggregation/aggregation.hpp:1318-1367):
    // M2 / MEDIAN / QUANTILE are double over arithmetic values (group_m2.cu
    // and group_quantiles.cu accept those only), NUNIQUE a size_type count,
    // NTH_ELEMENT the value's own type
    case GBX_AGG_M2:
    case GBX_AGG_MEDIAN:
    case GBX_AGG_QUANTILE:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_NUNIQUE: return GBX_TYPE_INT32;
    case GBX_AGG_NTH_ELEMENT: return t;
    default: return GBX_TYPE_EMPTY;
  }
}

// Kinds libcudf computes on its sort path (groupby/sort/aggregate.cpp) that
// are computed here by ordering each group's values (gbx_sort.cu); M2, also
// a sort-path kind there, comes from the hash table's shifted moments.
bool is_sort_kind(int32_t k)
{
  return k == GBX_AGG_MEDIAN || k == GBX_AGG_QUANTILE || k == GBX_AGG_NUNIQUE || k == GBX_AGG_NTH_ELEMENT;
}

// Kinds the batched form computes: the hash kinds but ARGMIN / ARGMAX.
bool is_batch_kind(int32_t k) { return is_hash_kind(k) && k != GBX_AGG_ARGMIN && k != GBX_AGG_ARGMAX; }

// Kinds libcudf accepts on its hash path (hash/groupby.cu:73-84).
bool is_hash_kind(int32_t k)
{
  switch (k) {
    case GBX_AGG_SUM:
    case GBX_AGG_PRODUCT:
    case GBX_AGG_MIN:
    case GBX_AGG_MAX:
    case GBX_AGG_ARGMIN:
    case GBX_AGG_ARGMAX:
    case GBX_AGG_COUNT_VALID:
    case GBX_AGG_COUNT_ALL:
    case GBX_AGG_SUM_OF_SQUARES:
    case GBX_AGG_MEAN:
    case GBX_AGG_STD:
    case GBX_AGG_VARIANCE: return true;
    default: return false;
  }
}

int32_t value_type(const gbx_column_view& c)
{
  if (c.type_id == GBX_TYPE_DICTIONARY32) return c.dict_keys ? c.dict_keys->type_id : GBX_TYPE_EMPTY;
  return c.type_id;
}

bool same_view(const gbx_column_view& a, const gbx_column_view& b)
{
  return a.type_id == b.type_id && a.size == b.size && a.offset == b.offset && a.data == b.data &&
         a.null_mask == b.null_mask && a.index_type_id == b.index_type_id && a.dict_keys == b.dict_keys &&
         a.scale == b.scale;
}

// -------------------------------------------------------------- allocation

void* Alloc::allocate(size_t bytes)
{
  if (bytes == 0) bytes = 8;
  bytes   = (bytes + 255) & ~size_t(255);
  void* p = nullptr;
  if (has_user) {
    p = user.allocate(user.ctx, bytes, st);
    if (!p) fail(GBX_ERR_ALLOC, "allocator returned null for %zu bytes", bytes);
    return p;
  }
  cudaError_t e = cudaMallocAsync(&p, bytes, st);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(GBX_ERR_ALLOC, "cudaMallocAsync(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  return p;
}

void Alloc::release(void* p, size_t bytes)
{
  if (!p) return;
  if (bytes == 0) bytes = 8;
  bytes = (bytes + 255) & ~size_t(255);
  if (has_user) user.deallocate(user.ctx, p, bytes, st);
  else cudaFreeAsync(p, st);
}

DeviceInfo current_device()
{
  DeviceInfo d;
  GBX_CUDA(cudaGetDevice(&d.device));
  GBX_CUDA(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, d.device));
  int optin = 0;
  GBX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.device));
  d.smem_optin = static_cast<size_t>(optin);
  int l2 = 0;
  GBX_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, d.device));
  d.l2_bytes = static_cast<size_t>(l2);
  return d;
}

uint64_t next_pow2(uint64_t v)
{
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace gbx

using namespace gbx;

// ------------------------------------------------------------- the object

struct gbx_groupby {
  std::vector<gbx_column_view> keys;
  std::vector<gbx_column_view> dict_keys;  // copies of each key column's dictionary keys
  int32_t null_policy = GBX_NULL_EXCLUDE;
  int32_t keys_are_sorted = 0;
  std::deque<std::vector<gbx_column_view>> members;  // copies of STRUCT keys' member views (and their offsets)
  int32_t strategy = GBX_STRATEGY_AUTO;
  int32_t timing = 0;
  cudaEvent_t events[6] = {};  // phase boundaries when timing is on
  int events_device = -1;
  gbx_stats stats{};
  ~gbx_groupby()
  {
    for (auto& e : events)
      if (e) cudaEventDestroy(e);
  }
};

int32_t gbx::groupby_strategy(const gbx_groupby* gb) { return gb->strategy; }

namespace {

constexpr int kMaxStructDepth = 4;

// Checks a STRUCT key column's members and points the view at copies of
// their descriptors held by the groupby (recursively, with STRING members'
// offsets), as the plain key descriptors are copied.
void adopt_struct_key(gbx_groupby* gb, gbx_column_view& v, int depth)
{
  GBX_EXPECTS(depth < kMaxStructDepth, "struct keys nested deeper than %d levels", kMaxStructDepth);
  GBX_EXPECTS(v.num_children > 0 && v.dict_keys != nullptr, "a STRUCT key column needs its members");
  gb->members.emplace_back(v.dict_keys, v.dict_keys + v.num_children);
  std::vector<gbx_column_view>& m = gb->members.back();
  for (gbx_column_view& c : m) {
    GBX_EXPECTS(c.offset >= 0 && c.size >= v.offset + v.size, "a struct member is shorter than its struct");
    if (c.type_id == GBX_TYPE_STRUCT) {
      adopt_struct_key(gb, c, depth + 1);
    } else if (c.type_id == GBX_TYPE_STRING) {
      GBX_EXPECTS(c.dict_keys != nullptr && (c.dict_keys->type_id == GBX_TYPE_INT32 ||
                                             c.dict_keys->type_id == GBX_TYPE_INT64),
                  "a STRING struct member needs its INT32 / INT64 offsets column");
      GBX_EXPECTS(c.dict_keys->size >= c.offset + c.size + 1, "offsets column too short");
      gb->members.emplace_back(1, *c.dict_keys);
      c.dict_keys = gb->members.back().data();
    } else if (!is_fixed_width(c.type_id) || c.type_id == GBX_TYPE_DICTIONARY32) {
      fail(GBX_ERR_UNSUPPORTED, "struct member type %d (list / dictionary / decimal128) is not supported",
           c.type_id);
    } else {
      c.num_children = 0;
      c.dict_keys    = nullptr;
    }
  }
  v.data      = nullptr;
  v.dict_keys = m.data();
}

}  // namespace

namespace gbx {
namespace {

// Records the phase boundaries of one aggregate() call on its stream.
struct PhaseTimer {
  gbx_groupby* gb;
  cudaStream_t st;
  bool on;
  PhaseTimer(gbx_groupby* g, cudaStream_t s, int device) : gb(g), st(s), on(g->timing != 0)
  {
    if (!on) return;
    if (gb->events_device != device) {
      for (auto& e : gb->events)
        if (e) cudaEventDestroy(e);
      for (auto& e : gb->events) GBX_CUDA(cudaEventCreate(&e));
      gb->events_device = device;
    }
  }
  void mark(int i)
  {
    if (on) GBX_CUDA(cudaEventRecord(gb->events[i], st));
  }
  // after the stream has been synchronised past mark(5)
  void read(gbx_stats& s)
  {
    if (!on) return;
    float t[5];
    for (int i = 0; i < 5; ++i) GBX_CUDA(cudaEventElapsedTime(&t[i], gb->events[i], gb->events[i + 1]));
    s.timed        = 1;
    s.sample_ms    = t[0];
    // phase 1 is the table fill, or the radix partition passes of the
    // partitioned strategy (which has no table to fill)
    const bool part = s.strategy == GBX_STRATEGY_PARTITIONED;
    s.init_ms       = part ? 0.f : t[1];
    s.partition_ms  = part ? t[1] : 0.f;
    s.aggregate_ms = t[2];
    s.compact_ms   = t[3];
    s.finalize_ms  = t[4];
    GBX_CUDA(cudaEventElapsedTime(&s.total_ms, gb->events[0], gb->events[5]));
  }
};

}  // namespace
}  // namespace gbx

namespace gbx {

// Output column allocation helper.
void alloc_column(Alloc& a, gbx_column& c, int32_t type_id, int32_t scale, int64_t n, bool with_mask)
{
  std::memset(&c, 0, sizeof(c));
  int w          = type_width(type_id == GBX_TYPE_DICTIONARY32 ? GBX_TYPE_INT32 : type_id);
  c.data_bytes   = static_cast<size_t>(n) * w;
  c.data         = n > 0 ? a.allocate(c.data_bytes) : nullptr;
  if (with_mask) {
    size_t words = static_cast<size_t>((n + 31) / 32);
    c.mask_bytes = ((words * 4 + 63) / 64) * 64;  // padded like cudf's bitmask allocations
    c.null_mask  = n > 0 ? static_cast<uint32_t*>(a.allocate(c.mask_bytes)) : nullptr;
  }
  c.view.type_id    = type_id;
  c.view.scale      = scale;
  c.view.size       = n;
  c.view.offset     = 0;
  c.view.data       = c.data;
  c.view.null_mask  = c.null_mask;
  c.view.null_count = with_mask ? -1 : 0;
}

bool is_count_kind(int32_t kind) { return kind == GBX_AGG_COUNT_VALID || kind == GBX_AGG_COUNT_ALL; }

bool counted_only(int32_t vt)
{
  return vt == GBX_TYPE_STRING || vt == GBX_TYPE_LIST || vt == GBX_TYPE_STRUCT || vt == GBX_TYPE_DECIMAL128;
}

void validate_requests(const gbx_request* reqs, int32_t nreq, int64_t n, bool count_any)
{
  GBX_EXPECTS(nreq >= 0 && (nreq == 0 || reqs != nullptr), "invalid request array");
  for (int32_t q = 0; q < nreq; ++q) {
    const gbx_request& r = reqs[q];
    // groupby.cu:210-214
    GBX_EXPECTS(r.values.size == n, "Size mismatch between request values and groupby keys.");
    GBX_EXPECTS(r.num_aggregations >= 0 && (r.num_aggregations == 0 || r.aggregations != nullptr),
                "invalid aggregation array");
    if (r.values.type_id == GBX_TYPE_DICTIONARY32)
      GBX_EXPECTS(r.values.dict_keys != nullptr, "dictionary column without keys");
    int32_t vt = value_type(r.values);
    for (int32_t k = 0; k < r.num_aggregations; ++k) {
      int32_t kind = r.aggregations[k].kind;
      // verify_valid_requests (groupby.cu:176-192)
      if (!is_hash_kind(kind) && !is_sort_kind(kind) && kind != GBX_AGG_M2) {
        if (kind == GBX_AGG_ANY || kind == GBX_AGG_ALL || kind > GBX_AGG_NTH_ELEMENT)
          fail(GBX_ERR_UNSUPPORTED,
               "aggregation kind %d is computed by libcudf's sort-based groupby only, and not by this library",
               kind);
        fail(GBX_ERR_LOGIC, "Invalid type/aggregation combination.");
      }
      const gbx_aggregation& ag = r.aggregations[k];
      if (kind == GBX_AGG_QUANTILE) {
        GBX_EXPECTS(ag.num_quantiles >= 0 && (ag.num_quantiles == 0 || ag.quantiles != nullptr),
                    "invalid quantile array");
        // select_quantile_data (quantiles_util.hpp:171-190) fails on others
        GBX_EXPECTS(ag.interpolation >= GBX_INTERP_LINEAR && ag.interpolation <= GBX_INTERP_NEAREST,
                    "Invalid interpolation operation for quantiles.");
      }
      if (kind == GBX_AGG_NUNIQUE || kind == GBX_AGG_NTH_ELEMENT)
        GBX_EXPECTS(ag.null_policy == GBX_NULL_EXCLUDE || ag.null_policy == GBX_NULL_INCLUDE,
                    "invalid null_policy %d", ag.null_policy);
      if (counted_only(vt)) {
        // COUNT reads only the rows' validity: any column type (hash/groupby.cu:73-84 with a size_type target)
        if (count_any && is_count_kind(kind)) continue;
        // MIN / MAX of strings: libcudf's sort path; here a best row per group
        if (count_any && vt == GBX_TYPE_STRING && (kind == GBX_AGG_MIN || kind == GBX_AGG_MAX)) {
          GBX_EXPECTS(r.values.dict_keys != nullptr && (r.values.dict_keys->type_id == GBX_TYPE_INT32 ||
                                                        r.values.dict_keys->type_id == GBX_TYPE_INT64),
                      "a STRING value column needs its INT32 / INT64 offsets column");
          GBX_EXPECTS(r.values.size == 0 || r.values.dict_keys->size >= r.values.offset + r.values.size + 1,
                      "offsets column too short");
          continue;
        }
        fail(GBX_ERR_UNSUPPORTED,
             "value type %d is aggregated by libcudf's sort-based groupby, which this library does not provide", vt);
      }
      GBX_EXPECTS(target_type(vt, kind) != GBX_TYPE_EMPTY, "Invalid type/aggregation combination.");
    }
  }
}

int64_t exact_null_count_or_neg(const gbx_column_view& c)
{
  if (c.null_mask == nullptr) return 0;
  return c.null_count;  // -1 when unknown
}

// Byte layout of one shared-memory table of S + 1 slots: keys, 8-byte
// accumulators, 4-byte accumulators, row counts.
SmemLayout make_smem_layout(const Plan& plan, uint32_t S)
{
  SmemLayout sl{};
  sl.slots     = S;
  uint32_t off = 0;
  sl.keys_off  = off;
  off += (S + 1) * plan.key.nwords * 8;
  for (int a = 0; a < plan.acc.nacc; ++a) {
    if (acc_bytes(plan.acc.kind[a]) == 8) {
      off           = (off + 7) & ~7u;
      sl.acc_off[a] = off;
      off += (S + 1) * 8;
    }
  }
  for (int a = 0; a < plan.acc.nacc; ++a) {
    if (acc_bytes(plan.acc.kind[a]) == 4) {
      sl.acc_off[a] = off;
      off += (S + 1) * 4;
    }
  }
  sl.rows_off = off;
  off += (S + 1) * 4;
  sl.total = (off + 15) & ~15u;
  return sl;
}

size_t slot_bytes(const Plan& plan)
{
  size_t b = static_cast<size_t>(plan.key.nwords) * 8 + 4;
  for (int a = 0; a < plan.acc.nacc; ++a) b += acc_bytes(plan.acc.kind[a]);
  return b;
}

// Builds the key plan.  `key_nulls[c]` is the null count of key column c.
KeyPlan make_key_plan(const gbx_column_view* keys, int nkeys, int32_t null_policy,
                      const std::vector<int64_t>& key_nulls, bool& ok)
{
  KeyPlan kp{};
  ok                   = true;
  kp.ncols             = nkeys;
  bool any_nulls       = false;
  for (auto v : key_nulls) any_nulls |= (v != 0);
  const bool include   = null_policy == GBX_NULL_INCLUDE;
  kp.skip_null_rows    = (!include && any_nulls) ? 1 : 0;
  // value fields first (never split across a word), then the null bits in
  // the first free bits of either word
  int word = 0, bit = 0;
  for (int c = 0; c < kp.ncols; ++c) {
    const gbx_column_view& col = keys[c];
    KeyCol& kc                 = kp.cols[c];
    int32_t phys_type          = col.type_id == GBX_TYPE_DICTIONARY32
                                   ? (col.index_type_id ? col.index_type_id : GBX_TYPE_INT32)
                                   : col.type_id;
    kc.data      = col.data;
    kc.mask      = key_nulls[c] != 0 ? col.null_mask : nullptr;
    kc.offset    = col.offset;
    kc.width     = static_cast<int8_t>(type_width(phys_type));
    kc.is_float  = is_floating(phys_type) ? 1 : 0;
    kc.is_bool   = phys_type == GBX_TYPE_BOOL8 ? 1 : 0;
    kc.null_bit  = (include && key_nulls[c] != 0) ? 1 : 0;
    kc.is_signed = (!is_unsigned(phys_type) && phys_type != GBX_TYPE_BOOL8) ? 1 : 0;
    int need     = kc.width * 8;
    if (bit + need > 64) {
      ++word;
      bit = 0;
    }
    if (word > 1) {
      ok = false;
      return kp;
    }
    kc.word  = static_cast<int8_t>(word);
    kc.shift = static_cast<int8_t>(bit);
    bit += need;
    kp.bits_used += need;
  }
  int used[2] = {word == 0 ? bit : 64, word == 1 ? bit : 0};
  int nwords  = word + 1;
  for (int c = 0; c < kp.ncols; ++c) {
    KeyCol& kc = kp.cols[c];
    if (!kc.null_bit) continue;
    int w = used[0] < 64 ? 0 : 1;
    if (w == 1 && used[1] >= 64) {
      ok = false;
      return kp;
    }
    nwords         = std::max(nwords, w + 1);
    kc.null_word   = static_cast<int8_t>(w);
    kc.null_shift  = static_cast<int8_t>(used[w]++);
    kp.bits_used  += 1;
  }
  kp.nwords = nwords;
  return kp;
}

std::vector<const gbx_column_view*> collect_channels(const gbx_request* reqs, int32_t nreq,
                                                     std::vector<int>& req_chan)
{
  req_chan.assign(nreq, -1);
  std::vector<const gbx_column_view*> chan_cols;
  for (int q = 0; q < nreq; ++q) {
    if (reqs[q].num_aggregations == 0) continue;
    int found = -1;
    for (size_t c = 0; c < chan_cols.size(); ++c)
      if (same_view(*chan_cols[c], reqs[q].values)) found = static_cast<int>(c);
    if (found < 0) {
      found = static_cast<int>(chan_cols.size());
      chan_cols.push_back(&reqs[q].values);
    }
    req_chan[q] = found;
  }
  if (static_cast<int>(chan_cols.size()) > kMaxChannels)
    fail(GBX_ERR_UNSUPPORTED, "more than %d distinct value columns in one call", kMaxChannels);
  return chan_cols;
}

void fill_channels(Plan& plan, const std::vector<const gbx_column_view*>& chan_cols,
                   const std::vector<int64_t>& chan_nulls, const gbx_request* reqs, int32_t nreq,
                   const std::vector<int>& req_chan)
{
  plan.nchan = static_cast<int32_t>(chan_cols.size());
  int nacc   = 0;
  auto add_acc = [&](int kind) -> int8_t {
    if (nacc >= kMaxAccs) fail(GBX_ERR_UNSUPPORTED, "too many accumulators in one call");
    plan.acc.kind[nacc] = static_cast<int8_t>(kind);
    return static_cast<int8_t>(nacc++);
  };
  for (int c = 0; c < plan.nchan; ++c) {
    const gbx_column_view& col = *chan_cols[c];
    Channel& ch                = plan.chan[c];
    std::memset(&ch, 0, sizeof(ch));
    ch.a_cnt = ch.a_sum = ch.a_min = ch.a_max = ch.a_sq = ch.a_k = ch.a_s2 = ch.a_prod = ch.a_amin = ch.a_amax = ch.a_s1 = -1;
    int32_t vt = value_type(col);
    ch.data    = col.data;
    ch.mask    = chan_nulls[c] != 0 ? col.null_mask : nullptr;
    ch.offset  = col.offset;
    if (col.type_id == GBX_TYPE_DICTIONARY32) {
      int32_t it     = col.index_type_id ? col.index_type_id : GBX_TYPE_INT32;
      ch.dict_data   = col.dict_keys->data;
      ch.dict_offset = col.dict_keys->offset;
      ch.dict_size   = col.dict_keys->size;
      ch.idx_width   = static_cast<int8_t>(type_width(it));
      ch.idx_signed  = is_unsigned(it) ? 0 : 1;
    }
    ch.ptype      = phys_of(vt);
    ch.is_float   = is_floating(vt) ? 1 : 0;
    uint32_t need = 0;
    for (int q = 0; q < nreq; ++q) {
      if (req_chan[q] != c) continue;
      for (int k = 0; k < reqs[q].num_aggregations; ++k) {
        switch (reqs[q].aggregations[k].kind) {
          case GBX_AGG_SUM: need |= N_SUM; break;
          case GBX_AGG_PRODUCT: need |= N_PROD; break;
          case GBX_AGG_MIN: need |= N_MIN; break;
          case GBX_AGG_MAX: need |= N_MAX; break;
          case GBX_AGG_ARGMIN: need |= N_AMIN; break;
          case GBX_AGG_ARGMAX: need |= N_AMAX; break;
          case GBX_AGG_COUNT_VALID: need |= N_CNT; break;
          case GBX_AGG_SUM_OF_SQUARES: need |= N_SQ; break;
          case GBX_AGG_MEAN: need |= N_SUM | N_CNT; break;
          case GBX_AGG_VARIANCE:
          case GBX_AGG_STD:
          case GBX_AGG_M2: need |= N_SUM | N_CNT | N_VAR; break;
          default: break;  // COUNT_ALL uses the row count
        }
      }
    }
    ch.need        = need;
    const bool m64 = ch.ptype == P_I64 || ch.ptype == P_U64 || ch.ptype == P_F64;
    // COUNT_VALID of a column without nulls is the group's row count; a
    // nullable column needs its own count (also the validity of SUM/MIN/...)
    if (chan_nulls[c] != 0) ch.a_cnt = add_acc(A_U32_ADD);
    if (need & N_SUM) ch.a_sum = add_acc(ch.is_float ? A_F64_ADD : A_I64_ADD);
    if (need & N_MIN) ch.a_min = add_acc(m64 ? A_U64_MIN : A_U32_MIN);
    if (need & N_MAX) ch.a_max = add_acc(m64 ? A_U64_MAX : A_U32_MAX);
    if (need & N_SQ) ch.a_sq = add_acc(ch.is_float ? A_F64_ADD : A_I64_ADD);
    if (need & N_PROD) ch.a_prod = add_acc(ch.is_float ? A_F64_MUL : A_I64_MUL);
    // ARGMIN / ARGMAX: a packed (value, row) word for values of up to 32
    // bits, a row index updated by compare-and-swap for 64-bit values
    if (need & N_AMIN) ch.a_amin = add_acc(m64 ? A_I32_ARGMIN_CAS : A_U64_ARGMIN);
    if (need & N_AMAX) ch.a_amax = add_acc(m64 ? A_I32_ARGMAX_CAS : A_U64_ARGMAX);
    if (need & N_VAR) {
      ch.a_k  = add_acc(A_F64_SHIFT);
      ch.a_s2 = add_acc(A_F64_ADD);
      if (ch.is_float) ch.a_s1 = add_acc(A_F64_ADD);
    }
  }
  plan.acc.nacc = nacc;
}

// Invert the expected distinct count of a uniform draw, d = C (1 - exp(-m / C)),
// then G = C (1 - exp(-N / C)).
namespace {
// Distinct keys expected among `rows` rows drawn uniformly from a population
// of C keys, where C is solved from `distinct` keys seen in `sampled` rows
// (D(m) = C (1 - e^{-m/C})).
double project_distinct(double sampled, double distinct, double rows)
{
  if (distinct >= sampled) return rows;
  double lo = distinct, hi = 1e12;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    double d   = mid * (1.0 - std::exp(-sampled / mid));
    if (d < distinct) lo = mid;
    else hi = mid;
  }
  const double C = 0.5 * (lo + hi);
  return C * (1.0 - std::exp(-rows / C));
}
}  // namespace

double estimate_groups(double sampled, double distinct, int64_t n, int64_t nsample)
{
  const double est = nsample >= n ? distinct : project_distinct(sampled, distinct, static_cast<double>(n));
  return std::max(1.0, std::min(est, static_cast<double>(n)));
}

double estimate_groups(double sampled, double distinct, double heavy, double heavy_rows, int64_t n, int64_t nsample)
{
  if (nsample >= n) return estimate_groups(sampled, distinct, n, nsample);
  const double light_sampled = sampled - heavy_rows, light_distinct = distinct - heavy;
  double est = heavy;
  if (light_sampled > 0 && light_distinct > 0)
    est += project_distinct(light_sampled, light_distinct, static_cast<double>(n) * (light_sampled / sampled));
  return std::max(1.0, std::min(est, static_cast<double>(n)));
}

}  // namespace gbx

namespace {

struct Call {
  gbx_groupby* gb;
  const gbx_request* reqs;
  int32_t nreq;
  gbx::Alloc alloc;
  gbx::DeviceInfo dev;
  int64_t n = 0;
};

void validate(const gbx_groupby* gb, const gbx_request* reqs, int32_t nreq, bool count_any = false)
{
  gbx::validate_requests(reqs, nreq, gb->keys.empty() ? 0 : gb->keys[0].size, count_any);
}

}  // namespace

// ================================================================== C ABI

extern "C" {

const char* gbx_last_error(void) { return g_last_error.c_str(); }
int32_t gbx_abi_version(void) { return GBX_ABI_VERSION; }
int32_t gbx_target_type(int32_t type_id, int32_t kind)
{
  if (!is_hash_kind(kind) && !is_sort_kind(kind) && kind != GBX_AGG_M2) return GBX_TYPE_EMPTY;
  return target_type(type_id, kind);
}

int gbx_groupby_create(const gbx_table_view* keys, int32_t null_policy, int32_t keys_are_sorted, gbx_groupby** out)
{
  return guarded([&] {
    GBX_EXPECTS(out != nullptr, "out is null");
    *out = nullptr;
    GBX_EXPECTS(keys != nullptr && keys->num_columns >= 0 && (keys->num_columns == 0 || keys->columns),
                "invalid keys table");
    GBX_EXPECTS(null_policy == GBX_NULL_EXCLUDE || null_policy == GBX_NULL_INCLUDE, "invalid null_policy");
    GBX_EXPECTS(keys_are_sorted == 0 || keys_are_sorted == 1, "invalid keys_are_sorted");
    auto* gb            = new gbx_groupby();
    gb->null_policy     = null_policy;
    gb->keys_are_sorted = keys_are_sorted;
    try {
      gb->keys.assign(keys->columns, keys->columns + keys->num_columns);
      gb->dict_keys.resize(gb->keys.size());
      for (size_t c = 0; c < gb->keys.size(); ++c) {
        gbx_column_view& k = gb->keys[c];
        GBX_EXPECTS(k.size == gb->keys[0].size, "key columns differ in size");
        if (k.type_id == GBX_TYPE_DICTIONARY32) {
          GBX_EXPECTS(k.dict_keys != nullptr, "dictionary key column without keys");
          gb->dict_keys[c] = *k.dict_keys;
          k.dict_keys      = &gb->dict_keys[c];
          int32_t it       = k.index_type_id ? k.index_type_id : GBX_TYPE_INT32;
          GBX_EXPECTS(is_integral(it) && it != GBX_TYPE_BOOL8, "dictionary indices must be integers");
        } else if (k.type_id == GBX_TYPE_STRING) {
          // characters in `data`, the offsets column in `dict_keys`
          GBX_EXPECTS(k.dict_keys != nullptr && (k.dict_keys->type_id == GBX_TYPE_INT32 ||
                                                 k.dict_keys->type_id == GBX_TYPE_INT64),
                      "a STRING key column needs its INT32 / INT64 offsets column");
          GBX_EXPECTS(k.size == 0 || k.dict_keys->size >= k.offset + k.size + 1, "offsets column too short");
          gb->dict_keys[c] = *k.dict_keys;
          k.dict_keys      = &gb->dict_keys[c];
        } else if (k.type_id == GBX_TYPE_STRUCT) {
          adopt_struct_key(gb, k, 0);
        } else if (!is_fixed_width(k.type_id)) {
          fail(GBX_ERR_UNSUPPORTED, "key type %d (list / decimal128) is not supported by this library", k.type_id);
        }
        GBX_EXPECTS(k.size >= 0 && k.offset >= 0, "negative size or offset");
        GBX_EXPECTS(k.size <= INT32_MAX, "row count exceeds cudf::size_type");
      }
    } catch (...) {
      delete gb;
      throw;
    }
    *out = gb;
  });
}

void gbx_groupby_destroy(gbx_groupby* gb) { delete gb; }

int gbx_groupby_set_strategy(gbx_groupby* gb, int32_t strategy)
{
  return guarded([&] {
    GBX_EXPECTS(gb != nullptr, "null groupby");
    GBX_EXPECTS(strategy == GBX_STRATEGY_AUTO || strategy == GBX_STRATEGY_PRIVATIZED ||
                  strategy == GBX_STRATEGY_GLOBAL || strategy == GBX_STRATEGY_WARP ||
                  strategy == GBX_STRATEGY_PARTITIONED || strategy == GBX_STRATEGY_BUCKETED,
                "strategy %d not available", strategy);
    gb->strategy = strategy;
  });
}

int gbx_groupby_set_timing(gbx_groupby* gb, int32_t enable)
{
  return guarded([&] {
    GBX_EXPECTS(gb != nullptr, "null groupby");
    gb->timing = enable ? 1 : 0;
  });
}

int gbx_groupby_last_stats(const gbx_groupby* gb, gbx_stats* out)
{
  return guarded([&] {
    GBX_EXPECTS(gb != nullptr && out != nullptr, "null argument");
    *out = gb->stats;
  });
}

int gbx_can_use_hash_groupby(const gbx_request* requests, int32_t num_requests)
{
  int rv = 1;
  int st = guarded([&] {
    GBX_EXPECTS(num_requests >= 0 && (num_requests == 0 || requests), "invalid request array");
    for (int32_t q = 0; q < num_requests; ++q) {
      int32_t vt = value_type(requests[q].values);
      if (vt == GBX_TYPE_STRUCT || vt == GBX_TYPE_LIST) rv = 0;
      for (int32_t k = 0; k < requests[q].num_aggregations; ++k) {
        int32_t kind = requests[q].aggregations[k].kind;
        if (!is_hash_kind(kind) || target_type(vt, kind) == GBX_TYPE_EMPTY) rv = 0;
      }
    }
  });
  return st == GBX_OK ? rv : -1;
}

void gbx_result_release(gbx_result* r)
{
  if (!r) return;
  auto* in = static_cast<ResultInternal*>(r->internal);
  auto free_col = [&](gbx_column& c) {
    if (in) {
      in->alloc.release(c.data, c.data_bytes);
      in->alloc.release(c.null_mask, c.mask_bytes);
    }
  };
  for (int c = 0; c < r->num_key_columns; ++c) free_col(r->keys[c]);
  if (in)
    for (auto& b : in->extra) in->alloc.release(b.first, b.second);
  for (int q = 0; q < r->num_requests; ++q) {
    for (int k = 0; k < r->requests[q].num_results; ++k) free_col(r->requests[q].results[k]);
    delete[] r->requests[q].results;
  }
  delete[] r->keys;
  delete[] r->requests;
  delete in;
  delete r;
}

int gbx_groupby_aggregate(gbx_groupby* gb,
                          const gbx_request* requests,
                          int32_t num_requests,
                          void* stream,
                          const gbx_allocator* mr,
                          gbx_result** out)
{
  gbx_result* res = nullptr;
  bool pack_args  = false;
  int st          = guarded([&] {
    GBX_EXPECTS(gb != nullptr && out != nullptr, "null argument");
    *out = nullptr;
    validate(gb, requests, num_requests, true);

    if (needs_string_extrema(requests, num_requests)) {
      // MIN / MAX of STRING values (gbx_rep.cu)
      if (gb->keys_are_sorted)
        fail(GBX_ERR_UNSUPPORTED, "MIN / MAX of STRING values with keys declared sorted are not provided");
      gb->stats = gbx_stats{};
      aggregate_string_extrema(gb, gb->keys, gb->null_policy, requests, num_requests, stream, mr, &res, &gb->stats);
      return;
    }
    if (needs_count_stand_ins(requests, num_requests)) {
      // COUNT of STRING / LIST / STRUCT / DECIMAL128 values (gbx_args.cu)
      aggregate_with_count_stand_ins(gb, gb->keys.empty() ? 0 : gb->keys[0].size, requests, num_requests, stream,
                                     mr, &res);
      return;
    }
    if (gb->keys_are_sorted) {
      // keys the caller declares sorted group by runs (gbx_rep.cu)
      gb->stats = gbx_stats{};
      aggregate_presorted(gb, gb->keys, gb->null_policy, requests, num_requests, stream, mr, &res, &gb->stats);
      return;
    }
    if (keys_need_representatives(gb->keys, gb->null_policy)) {
      // STRING keys, or keys beyond two packed 64-bit words (gbx_rep.cu)
      gb->stats = gbx_stats{};
      aggregate_by_representatives(gb, gb->keys, gb->null_policy, requests, num_requests, stream, mr, &res,
                                   &gb->stats);
      return;
    }
    Call call{gb, requests, num_requests};
    call.alloc.st = static_cast<cudaStream_t>(stream);
    if (mr && mr->allocate && mr->deallocate) {
      call.alloc.user     = *mr;
      call.alloc.has_user = true;
    }
    call.dev = current_device();
    call.n   = gb->keys.empty() ? 0 : gb->keys[0].size;
    cudaStream_t s = call.alloc.st;
    const int nkeys = static_cast<int>(gb->keys.size());

    res                  = new gbx_result();
    std::memset(res, 0, sizeof(*res));
    auto* internal       = new ResultInternal{call.alloc};
    res->internal        = internal;
    res->num_key_columns = nkeys;
    res->num_requests    = num_requests;
    res->keys            = new gbx_column[nkeys > 0 ? nkeys : 1]();
    res->requests        = new gbx_aggregation_result[num_requests > 0 ? num_requests : 1]();
    for (int q = 0; q < num_requests; ++q) {
      res->requests[q].num_results = requests[q].num_aggregations;
      res->requests[q].results     = new gbx_column[requests[q].num_aggregations > 0 ? requests[q].num_aggregations : 1]();
    }

    gb->stats          = gbx_stats{};
    gb->stats.num_rows = call.n;

    // ---- distinct value columns -> channels
    std::vector<int> req_chan;
    std::vector<const gbx_column_view*> chan_cols = collect_channels(requests, num_requests, req_chan);

    // ---- null counts (one small kernel + one read, merged with the sample read)
    std::vector<int64_t> key_nulls(nkeys, 0), chan_nulls(chan_cols.size(), 0);
    MaskSpans ms{};
    std::vector<std::pair<int, int>> span_owner;  // (0=key,1=chan, index)
    for (int c = 0; c < nkeys; ++c) {
      int64_t v = exact_null_count_or_neg(gb->keys[c]);
      key_nulls[c] = v;
      if (v < 0) {
        ms.span[ms.n++] = MaskSpan{gb->keys[c].null_mask, gb->keys[c].offset, gb->keys[c].size};
        span_owner.push_back({0, c});
      }
    }
    for (size_t c = 0; c < chan_cols.size(); ++c) {
      int64_t v     = exact_null_count_or_neg(*chan_cols[c]);
      chan_nulls[c] = v;
      if (v < 0) {
        ms.span[ms.n++] = MaskSpan{chan_cols[c]->null_mask, chan_cols[c]->offset, chan_cols[c]->size};
        span_owner.push_back({1, static_cast<int>(c)});
      }
    }

    // ---- empty input: typed empty results (groupby.cu:150-172, 218)
    if (call.n == 0) {
      for (int c = 0; c < nkeys; ++c) {
        alloc_column(call.alloc, res->keys[c], gb->keys[c].type_id, gb->keys[c].scale, 0, false);
        if (gb->keys[c].type_id == GBX_TYPE_DICTIONARY32) {
          res->keys[c].view.dict_keys     = gb->keys[c].dict_keys;
          res->keys[c].view.index_type_id = GBX_TYPE_INT32;
        }
      }
      for (int q = 0; q < num_requests; ++q) {
        int32_t vt = value_type(requests[q].values);
        for (int k = 0; k < requests[q].num_aggregations; ++k) {
          int32_t tt = target_type(vt, requests[q].aggregations[k].kind);
          alloc_column(call.alloc, res->requests[q].results[k], tt, is_decimal(tt) ? requests[q].values.scale : 0, 0,
                       false);
        }
      }
      return;
    }

    Scratch scratch(&call.alloc);
    PhaseTimer timer(gb, s, call.dev.device);
    int launches = 0;
    timer.mark(0);
    // control block: [0..1] sample counters, [2..25] valid counts, [26] status,
    // [27] num_selected, [28..31] partitioned-path counters, [32..33] heavy keys
    // of the sample and their rows
    constexpr int kCtlWords = 34;
    auto* ctl = static_cast<unsigned long long*>(scratch.get(kCtlWords * 8));
    GBX_CUDA(cudaMemsetAsync(ctl, 0, kCtlWords * 8, s));
    int32_t* d_status        = reinterpret_cast<int32_t*>(ctl + 26);
    int64_t* d_num_selected  = reinterpret_cast<int64_t*>(ctl + 27);
    GBX_CUDA(launch_count_valid(ms, ctl + 2, call.dev.num_sms, s));
    launches += ms.n > 0 ? 1 : 0;

    bool key_ok       = true;
    KeyPlan kp_sample =
      make_key_plan(gb->keys.data(), nkeys, gb->null_policy, std::vector<int64_t>(nkeys, -1), key_ok);
    if (!key_ok)
      fail(GBX_ERR_UNSUPPORTED, "key columns need more than 128 packed bits; wider composite keys are not supported");

    // ---- sampled distinct count
    const int64_t nsample = std::min<int64_t>(call.n, 1 << 16);
    const uint64_t set_cap = 1 << 18;
    auto* set      = static_cast<uint64_t*>(scratch.get(set_cap * 8));
    auto* set_rows = static_cast<uint32_t*>(scratch.get(set_cap * 4));
    GBX_CUDA(launch_sample(kp_sample, call.n, nsample, set, set_rows, set_cap, ctl, ctl + 32, call.dev.num_sms, s));
    launches += 3;
    timer.mark(1);

    unsigned long long h_ctl[kCtlWords];
    GBX_CUDA(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < span_owner.size(); ++i) {
      int64_t nulls = static_cast<int64_t>(ms.span[i].size) - static_cast<int64_t>(h_ctl[2 + i]);
      if (span_owner[i].first == 0) key_nulls[span_owner[i].second] = nulls;
      else chan_nulls[span_owner[i].second] = nulls;
    }
    double est = estimate_groups(static_cast<double>(h_ctl[0]), static_cast<double>(h_ctl[1]),
                                 static_cast<double>(h_ctl[32]), static_cast<double>(h_ctl[33]), call.n, nsample);
    gb->stats.estimated_groups = static_cast<int64_t>(est);

    // ---- plan
    Plan plan{};
    plan.key = make_key_plan(gb->keys.data(), nkeys, gb->null_policy, key_nulls, key_ok);
    fill_channels(plan, chan_cols, chan_nulls, requests, num_requests, req_chan);
    const int nacc = plan.acc.nacc;

    // ---- strategy and sizes
    const size_t slot_bytes  = gbx::slot_bytes(plan);
    const size_t smem_budget = std::min<size_t>(call.dev.smem_optin, 100 * 1024);
    uint32_t s_max           = 1;
    while (static_cast<size_t>(s_max * 2 + 1) * slot_bytes + 16 * (nacc + 2) <= smem_budget && s_max < (1u << 16))
      s_max *= 2;
    // warp-private tables: 8 warps per CTA, each with a table at load <= ~0.8
    uint32_t s_warp = 32;
    while (s_warp * 0.8 < est && s_warp < (1u << 14)) s_warp *= 2;
    const bool warp_fits = static_cast<size_t>(8) * make_smem_layout(plan, s_warp).total <= 200 * 1024;
    uint64_t cap = next_pow2(static_cast<uint64_t>(std::max(2.0 * est, 1024.0)));
    cap          = std::min<uint64_t>(cap, 1ULL << 31);
    // the global table stays (mostly) resident in L2 while the rows stream
    // through: at 3e5 groups (a 92 MB table) it still ran 13.0 ms against the
    // partitioned path's 19.5 ms
    const bool global_in_l2 =
      static_cast<double>(cap + 1) * static_cast<double>(slot_bytes) <= static_cast<double>(call.dev.l2_bytes);
    // BUCKETED: one radix pass into 2^8 buckets (two passes, 2^16, when a
    // bucket holds too many groups), then the tiled kernel over contiguous
    // runs of the bucket-ordered rows, one run per CTA (two CTAs per SM): a run
    // meets about est / runs groups plus those of the bucket or two it cuts,
    // which must fit a tiled table at load <= 1/2
    // (below kBucketedMinRows rows the partitioning costs more than the global
    // table's atomics it saves)
    constexpr int64_t kBucketedMinRows = int64_t(1) << 22;
    int bucket_bits       = 0;
    uint32_t bucket_slots = 0;
    for (int bb : {8, 16}) {
      const double groups = est / (2.0 * call.dev.num_sms) + est / static_cast<double>(1u << bb);
      const auto Sb = static_cast<uint32_t>(next_pow2(static_cast<uint64_t>(std::max(2.0 * groups, 64.0))));
      if (Sb <= 1024 && tiled_fits(make_smem_layout(plan, Sb), plan.nchan)) {
        bucket_bits  = bb;
        bucket_slots = Sb;
        break;
      }
    }
    int strategy = gb->strategy;
    if (strategy == GBX_STRATEGY_BUCKETED && bucket_bits == 0) {
      // forced with more groups than a tiled table holds: the largest table
      // that fits (rows of groups beyond it go to the global table directly)
      bucket_bits = 16;
      for (uint32_t Sb = 1024; Sb >= 64 && bucket_slots == 0; Sb >>= 1)
        if (tiled_fits(make_smem_layout(plan, Sb), plan.nchan)) bucket_slots = Sb;
      if (bucket_slots == 0) strategy = GBX_STRATEGY_GLOBAL;
    }
    // Skewed keys: when the keys sampled 4 or more times hold most sampled
    // rows and fit a CTA table of the streamed-tile kernel, that kernel keeps
    // them in shared memory and sends the rare keys' rows to the global table
    // (a Zipf key whose hottest group holds a fifth of the rows would
    // otherwise serialise the global table's atomics on one slot).
    const double s_heavy = static_cast<double>(h_ctl[32]), s_heavy_rows = static_cast<double>(h_ctl[33]);
    const bool skewed    = h_ctl[0] > 0 && s_heavy_rows >= 0.75 * static_cast<double>(h_ctl[0]);
    // table of the streamed-tile kernel: twice the heavy keys (one CTA an SM
    // when it does not fit two)
    uint32_t stream_slots = 0;
    if (skewed && plan.key.nwords == 1 && !plan_has_arg(plan)) {
      const auto need = static_cast<uint32_t>(next_pow2(static_cast<uint64_t>(std::max(2.0 * s_heavy, 64.0))));
      if (need <= 4096 && stream_fits(plan, make_smem_layout(plan, need))) stream_slots = need;
    }
    bool skew_stream = false;
    if (strategy == GBX_STRATEGY_AUTO) {
      // measured on B200 (100M rows, 12 accumulators): at 100 groups the shared
      // table with 32/64-bit shared atomics 4.0 ms, warp-private tables 7.2 ms;
      // at 1e4 groups the L2-resident global table 9.4 ms, the partitioned
      // path 21.4 ms; at 1e6 groups (table beyond L2) 32.6 ms against 17.2 ms
      if (est * 2.0 <= static_cast<double>(s_max)) strategy = GBX_STRATEGY_PRIVATIZED;
      else if (stream_slots > 0) {
        strategy    = GBX_STRATEGY_PRIVATIZED;
        skew_stream = true;
        // the rare keys land in the global table: room for more of them than
        // the sample saw
        cap = std::min<uint64_t>(cap * 4, 1ULL << 31);
      } else if (warp_fits) strategy = GBX_STRATEGY_WARP;
      else if (global_in_l2)
        strategy = bucket_bits > 0 && call.n >= kBucketedMinRows ? GBX_STRATEGY_BUCKETED : GBX_STRATEGY_GLOBAL;
      else strategy = GBX_STRATEGY_PARTITIONED;
    }
    if (strategy == GBX_STRATEGY_WARP && !warp_fits) strategy = GBX_STRATEGY_PRIVATIZED;
    // ARGMIN / ARGMAX record each row's own index where it is accumulated:
    // only the kernels that read the caller's rows in place (the privatised
    // shared table, untiled, and the global table) do
    const bool arg_kinds = plan_has_arg(plan);
    if (arg_kinds && strategy != GBX_STRATEGY_PRIVATIZED && strategy != GBX_STRATEGY_GLOBAL) {
      if (args_packable(requests, num_requests)) {
        // values of up to 32 bits: the ARG kinds become MIN / MAX of packed
        // words that every strategy computes (gbx_args.cu); this call is
        // redone with those requests
        pack_args = true;
        return;
      }
      strategy = est * 2.0 <= static_cast<double>(s_max) ? GBX_STRATEGY_PRIVATIZED : GBX_STRATEGY_GLOBAL;
    }
    // MEDIAN / QUANTILE / NUNIQUE / NTH_ELEMENT label each row by a probe of
    // the finished global table, which the partitioned path does not build
    bool has_sorted = false;
    for (int q = 0; q < num_requests; ++q)
      for (int k = 0; k < requests[q].num_aggregations; ++k)
        has_sorted = has_sorted || is_sort_kind(requests[q].aggregations[k].kind);
    if (has_sorted && strategy == GBX_STRATEGY_PARTITIONED) strategy = GBX_STRATEGY_GLOBAL;

    gb->stats.strategy = strategy;

    // Allocates the key and result columns with room for `rows` groups and
    // describes them for the kernels.
    // (the sorted kinds' columns are listed in `sorted_outs`, with the index
    // of their null counter, and written after the finalize kernel)
    std::vector<SortedOut> sorted_outs;
    std::vector<int> sorted_out_index;
    std::vector<double> h_quantiles;
    auto build_outputs = [&](int64_t rows) -> OutPlan {
      OutPlan op{};
      sorted_outs.clear();
      sorted_out_index.clear();
      h_quantiles.clear();
      for (int c = 0; c < nkeys; ++c) {
        const gbx_column_view& kcv = gb->keys[c];
        bool with_mask             = plan.key.cols[c].null_bit != 0;
        alloc_column(call.alloc, res->keys[c], kcv.type_id, kcv.scale, rows, with_mask);
        if (kcv.type_id == GBX_TYPE_DICTIONARY32) {
          int32_t it = kcv.index_type_id ? kcv.index_type_id : GBX_TYPE_INT32;
          res->keys[c].view.index_type_id = it;
          res->keys[c].view.dict_keys     = kcv.dict_keys;
          if (type_width(it) != 4) {
            // re-allocate data at the index width
            call.alloc.release(res->keys[c].data, res->keys[c].data_bytes);
            res->keys[c].data_bytes = static_cast<size_t>(rows) * type_width(it);
            res->keys[c].data       = rows > 0 ? call.alloc.allocate(res->keys[c].data_bytes) : nullptr;
            res->keys[c].view.data  = res->keys[c].data;
          }
        }
        if (with_mask) res->keys[c].view.null_count = -1;
        op.key_data[c] = res->keys[c].data;
        op.key_mask[c] = res->keys[c].null_mask;
      }
      for (int q = 0; q < num_requests; ++q) {
        const gbx_request& r = requests[q];
        int32_t vt           = value_type(r.values);
        for (int k = 0; k < r.num_aggregations; ++k) {
          const gbx_aggregation& ag = r.aggregations[k];
          int32_t kind   = ag.kind;
          int32_t tt     = target_type(vt, kind);
          bool has_nulls = chan_nulls[req_chan[q]] != 0;
          // nullable iff the values have nulls; COUNT never; VAR/STD always
          // (hash/groupby.cu:424-454); QUANTILE / MEDIAN always
          // (group_quantiles.cu); NTH_ELEMENT while some output is null (the
          // mask is dropped below when none is, as group_nth_element.cu
          // does); NUNIQUE never (group_nunique.cu)
          bool with_mask = (kind == GBX_AGG_COUNT_VALID || kind == GBX_AGG_COUNT_ALL || kind == GBX_AGG_NUNIQUE)
                             ? false
                             : (has_nulls || kind == GBX_AGG_VARIANCE || kind == GBX_AGG_STD ||
                                kind == GBX_AGG_QUANTILE || kind == GBX_AGG_MEDIAN || kind == GBX_AGG_NTH_ELEMENT);
          int32_t scale  = is_decimal(tt) ? (r.values.type_id == GBX_TYPE_DICTIONARY32 ? r.values.dict_keys->scale
                                                                                       : r.values.scale)
                                          : 0;
          // QUANTILE: num_quantiles rows per group
          const int64_t nq = kind == GBX_AGG_QUANTILE ? ag.num_quantiles : 1;
          gbx_column& oc   = res->requests[q].results[k];
          alloc_column(call.alloc, oc, tt, scale, rows * nq, with_mask);
          if (op.nout >= kMaxOut) fail(GBX_ERR_UNSUPPORTED, "more than %d results in one call", kMaxOut);
          if (is_sort_kind(kind)) {
            SortedOut so{};
            so.kind          = kind;
            so.chan          = req_chan[q];
            so.null_policy   = ag.null_policy;
            so.interpolation = kind == GBX_AGG_MEDIAN ? GBX_INTERP_LINEAR : ag.interpolation;
            so.num_quantiles = static_cast<int32_t>(nq);
            so.out_width     = type_width(tt);
            so.nth           = ag.ddof;
            so.data          = oc.data;
            so.mask          = oc.null_mask;
            // offset of this output's quantiles in h_quantiles until uploaded
            so.quantiles_dev = reinterpret_cast<const double*>(static_cast<uintptr_t>(h_quantiles.size()));
            if (kind == GBX_AGG_MEDIAN) h_quantiles.push_back(0.5);
            else if (kind == GBX_AGG_QUANTILE) h_quantiles.insert(h_quantiles.end(), ag.quantiles, ag.quantiles + nq);
            sorted_outs.push_back(so);
            sorted_out_index.push_back(op.nout);
          }
          OutCol& o   = op.out[op.nout++];
          o.data      = is_sort_kind(kind) ? nullptr : oc.data;
          o.mask      = oc.null_mask;
          o.kind      = kind;
          o.ddof      = r.aggregations[k].ddof;
          o.chan      = static_cast<int8_t>(req_chan[q]);
          o.out_ptype = phys_of(tt);
          o.out_width = static_cast<int8_t>(type_width(tt));
        }
      }
      return op;
    };
    // every output column, keys first, in request order
    auto for_each_output = [&](auto&& fn) {
      for (int c = 0; c < nkeys; ++c) fn(res->keys[c], c);
      int o = 0;
      for (int q = 0; q < num_requests; ++q)
        for (int k = 0; k < requests[q].num_aggregations; ++k, ++o) fn(res->requests[q].results[k], kMaxKeyCols + o);
    };

    // bucket-ordered copies of the rows (radix partitioning): packed key
    // words, resolved value bits, a validity byte per row of a nullable channel
    auto part_bufs = [&]() {
      PartBufs pb{};
      for (int w = 0; w < plan.key.nwords; ++w)
        pb.keys[w] = static_cast<const uint64_t*>(scratch.get(static_cast<size_t>(call.n) * 8));
      for (int c = 0; c < plan.nchan; ++c) {
        const int width = pt_width(plan.chan[c].ptype);
        pb.col[c].width = width;
        pb.col[c].vals  = scratch.get(static_cast<size_t>(call.n) * width);
        pb.col[c].valid =
          plan.chan[c].a_cnt >= 0 ? static_cast<const uint8_t*>(scratch.get(static_cast<size_t>(call.n))) : nullptr;
      }
      return pb;
    };

    if (strategy == GBX_STRATEGY_PARTITIONED) {
      // ---- radix-partitioned path (gbx_part.cu)
      // warp table slots (two CTAs per SM), halved until eight warps' tables
      // and scratch fit one CTA's shared memory (wide schemas)
      uint32_t S    = slot_bytes >= 48 ? 128u : 256u;
      SmemLayout sl = make_smem_layout(plan, S);
      auto part_smem = [&]() { return static_cast<size_t>(sl.total) * 8 + 8 * (S + 32) * 4; };
      while (S > 32 && part_smem() > call.dev.smem_optin) {
        S >>= 1;
        sl = make_smem_layout(plan, S);
      }
      if (part_smem() > call.dev.smem_optin)
        fail(GBX_ERR_UNSUPPORTED, "per-group state too large for the partitioned path");
      // target groups per bucket: half the table, so that the fullest of ~1M
      // buckets (mean + 5 sigma of a Poisson count) still fits
      const double gpb  = S * 0.5;
      int bits          = 0;
      while (static_cast<double>(1ull << bits) * gpb < est && bits < 22) ++bits;
      // one table per CTA instead (up to 4,096 slots, ~2,048 groups per
      // bucket) from 2^9 such buckets on: where that needs fewer 8-bit radix
      // passes than warp tables do, the bucket count is rounded up to whole
      // passes (smaller buckets, same passes), else it stays the warp tables'
      // (measured at 1e6 groups in 100M rows, 2^14 buckets: grouping and folds
      // 3.4 ms with CTA tables against 5.6 ms with warp tables; at 1e8, 2^16
      // buckets of 256-2,048 slots ran 9.2 ms against 10.5 ms for 2^15 of
      // 4,096); the table is sized for twice a bucket's mean groups
      const int warp_bits = bits;
      int cta_bits        = 0;
      while (static_cast<double>(1ull << cta_bits) * 2048.0 < est && cta_bits < 22) ++cta_bits;
      bool cta_rank  = false;
      uint32_t S_cta = 0;
      if (cta_bits >= 9 && (cta_bits + 7) / 8 <= (warp_bits + 7) / 8) {
        cta_rank = true;
        bits     = (cta_bits + 7) / 8 < (warp_bits + 7) / 8 ? 8 * ((cta_bits + 7) / 8) : warp_bits;
        S_cta    = static_cast<uint32_t>(
          std::min<uint64_t>(next_pow2(static_cast<uint64_t>(std::max(2.0 * est / static_cast<double>(1ull << bits), 256.0))),
                             4096));
      }
      PartBufs pbufs = part_bufs();
      // the radix passes' second set of copies and their counters
      PartBufs tbufs{};
      uint32_t* rcounts  = nullptr;
      uint32_t* roffsets = nullptr;
      void* rtemp        = nullptr;
      size_t rtemp_bytes = 0;
      uint32_t* n_kept   = nullptr;  // rows the radix passes keep (device)
      uint2* group_runs  = nullptr;  // (first sorted row, rows) per output row
      // outputs sized for the upper bound (every row its own group): the group
      // count is only known once the buckets have been written out
      OutPlan pop    = build_outputs(call.n);
      auto* p_nulls  = static_cast<unsigned long long*>(scratch.get((kMaxKeyCols + kMaxOut) * 8));
      pop.null_counts = p_nulls;
      int64_t Gp = 0;
      for (int attempt = 0;; ++attempt) {
        const uint32_t P = 1u << bits;
        PartPlan pp{};
        pp.bits         = bits;
        pp.shard_bits   = std::max(0, std::min(5, 12 - bits));
        // whole buckets up to the rows whose ranks fit a record: 16 bits beside
        // a warp table's slot, 19 beside a CTA table's
        pp.slice_rows = cta_rank ? (1u << 19) : 16384;
        pp.region_slots = S;
        pp.status       = d_status;
        auto arr        = [&]() { return static_cast<uint32_t*>(scratch.get((static_cast<size_t>(P) + 1) * 4)); };
        const size_t nctr = (static_cast<size_t>(P) << pp.shard_bits) + 1;
        pp.counts       = static_cast<uint32_t*>(scratch.get(nctr * 4));
        pp.offsets      = static_cast<uint32_t*>(scratch.get(nctr * 4));
        pp.cursor       = static_cast<uint32_t*>(scratch.get(nctr * 4));
        pp.nslices      = arr();
        pp.item_start   = arr();
        pp.multi        = arr();
        pp.region       = arr();
        pp.item_bucket  = nullptr;
        pp.item_counter = ctl + 29;
        pp.out_counter  = ctl + 30;
        GBX_CUDA(cudaMemsetAsync(ctl + 26, 0, 6 * 8, s));  // status, counters, special flag
        for_each_output([&](gbx_column& c, int) {
          if (c.null_mask) GBX_CUDA(cudaMemsetAsync(c.null_mask, 0, c.mask_bytes, s));
        });
        GBX_CUDA(cudaMemsetAsync(p_nulls, 0, (kMaxKeyCols + kMaxOut) * 8, s));
        // many buckets: coalesced radix passes (gbx_radix.cu), whose first
        // histogram also counts the rows per bucket
        const bool use_radix = pp.shard_bits == 0 && bits >= 9;
        size_t temp_bytes    = 0;
        GBX_CUDA(launch_part_layout(pp, nullptr, &temp_bytes, call.dev.num_sms, s));
        void* temp = scratch.get(temp_bytes);
        if (use_radix) {
          // the rows go to bucket order first; the bucket offsets are then
          // read off the partitioned keys (no per-row counter atomics)
          if (rcounts == nullptr) {
            tbufs    = part_bufs();
            rcounts  = static_cast<uint32_t*>(scratch.get(part_radix_count_bytes(call.n)));
            roffsets = static_cast<uint32_t*>(scratch.get(part_radix_count_bytes(call.n)));
            GBX_CUDA(part_radix_temp_bytes(call.n, &rtemp_bytes));
            rtemp  = scratch.get(rtemp_bytes);
            n_kept = static_cast<uint32_t*>(scratch.get(sizeof(uint32_t)));
          }
          GBX_CUDA(launch_part_radix_hist0(plan, call.n, bits, rcounts, nullptr, s));
          GBX_CUDA(launch_part_radix(plan, call.n, bits, n_kept, pbufs, tbufs, rcounts, roffsets, rtemp, rtemp_bytes,
                                     d_status, /*hist0_done=*/true, s));
          GBX_CUDA(launch_part_bounds(plan.key.nwords, pbufs.keys, n_kept, bits, pp.offsets, call.dev.num_sms, s));
          GBX_CUDA(launch_part_layout(pp, temp, &temp_bytes, call.dev.num_sms, s, /*offsets_ready=*/true));
          // first histogram, 3 launches per pass (the first: scan, kept rows,
          // scatter), bounds, slices + 2 scans
          launches += 1 + 3 * ((bits + 7) / 8) + 1 + 3;
        } else {
          GBX_CUDA(launch_part_hist(plan.key, call.n, pp, call.dev.num_sms, s));
          GBX_CUDA(launch_part_layout(pp, temp, &temp_bytes, call.dev.num_sms, s));
          launches += 5;  // histogram, scan, slices, 2 scans
        }
        uint32_t h_counts[2] = {0, 0};  // regions, work items
        GBX_CUDA(cudaMemcpyAsync(&h_counts[0], pp.region + P, 4, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaMemcpyAsync(&h_counts[1], pp.item_start + P, 4, cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaStreamSynchronize(s));
        const uint32_t h_regions = h_counts[0];  // buckets larger than slice_rows
        const uint32_t h_items   = h_counts[1];  // their slices
        // region tables of the buckets split over several warps
        TableRef t2{};
        if (h_items > 0) {
          pp.item_bucket = static_cast<uint32_t*>(scratch.get((static_cast<size_t>(h_items) + 1) * 4));
          GBX_CUDA(launch_part_items(pp, call.n, call.dev.num_sms, s));
          t2.cap  = static_cast<uint64_t>(h_regions) * S;
          t2.keys = static_cast<uint64_t*>(scratch.get((t2.cap + 1) * plan.key.nwords * 8));
          t2.rows = static_cast<uint32_t*>(scratch.get((t2.cap + 1) * 4));
          for (int a = 0; a < nacc; ++a) t2.acc[a] = scratch.get((t2.cap + 1) * acc_bytes(plan.acc.kind[a]));
          t2.special_used = reinterpret_cast<uint32_t*>(ctl + 28);
          t2.status       = d_status;
          GBX_CUDA(launch_init_table(t2, plan.acc, plan.key.nwords, call.dev.num_sms, s));
          launches += 2;
        }
        if (!use_radix) {
          GBX_CUDA(launch_part_scatter(plan, call.n, pp, pbufs, call.dev.num_sms, s));
          launches += 1;
          if (tbufs.keys[0] == nullptr) tbufs = part_bufs();
        }
        // the second set of copies (free again after the radix passes) takes
        // the whole buckets' rows in group order; its key words hold the rank
        // records of buckets too large for shared memory
        pp.rank_rec       = const_cast<uint32_t*>(reinterpret_cast<const uint32_t*>(tbufs.keys[0]));
        pp.bucket_counter = ctl + 31;
        if (group_runs == nullptr) group_runs = static_cast<uint2*>(scratch.get(static_cast<size_t>(call.n) * 8));
        pp.group_run = group_runs;
        timer.mark(2);
        if (cta_rank) GBX_CUDA(launch_part_ranked_cta(plan, pp, pbufs, tbufs, S_cta, pop, call.dev.num_sms, s));
        else GBX_CUDA(launch_part_ranked(plan, pp, pbufs, tbufs, S, pop, call.dev.num_sms, s));
        launches += 1 + plan.nchan;  // grouping, one fold per value channel
        if (h_items > 0) {
          GBX_CUDA(launch_part_agg(plan, pp, pbufs, t2, sl, call.dev.num_sms, s));
          timer.mark(3);
          GBX_CUDA(launch_part_region_finalize(plan, pp, t2, pop, call.dev.num_sms, s));
          launches += 2;
        } else {
          timer.mark(3);
        }
        timer.mark(4);
        GBX_CUDA(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
        GBX_CUDA(cudaStreamSynchronize(s));
        int32_t status;
        std::memcpy(&status, reinterpret_cast<char*>(h_ctl) + 26 * 8, 4);
        Gp = static_cast<int64_t>(h_ctl[30]);
        if (status & S_SPIN_LIMIT) fail(GBX_ERR_DEVICE, "a bounded device loop gave up (status 0x%x)", status);
        if (status & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");
        if (status & S_CHECK_FAILED) fail(GBX_ERR_DEVICE, "partitioned path: rows out of bucket order (status 0x%x)", status);
        if ((status & S_TABLE_FULL) == 0) {
          gb->stats.table_capacity = static_cast<int64_t>(P) * (cta_rank ? S_cta : S);
          gb->stats.partition_bits = bits;
          gb->stats.bucket_slots   = static_cast<int32_t>(cta_rank ? S_cta : S);
          break;
        }
        // a bucket held more groups than its table: warp tables (whose slices
        // of very large buckets merge through their own region tables) at
        // their own bucket count or 4x the failed one, else 4x the buckets
        if (attempt >= 3 || bits >= 24) fail(GBX_ERR_DEVICE, "partitioned aggregation overflow at %u buckets", P);
        gb->stats.retries++;
        if (cta_rank) {
          cta_rank = false;
          bits     = std::max(warp_bits, bits + 2);
        } else {
          bits += 2;
        }
      }
      timer.mark(5);
      std::vector<unsigned long long> h_nulls(kMaxKeyCols + kMaxOut, 0);
      GBX_CUDA(cudaMemcpyAsync(h_nulls.data(), p_nulls, h_nulls.size() * 8, cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      for_each_output([&](gbx_column& c, int idx) {
        c.view.size = Gp;
        if (c.null_mask) c.view.null_count = static_cast<int64_t>(h_nulls[idx]);
      });
      res->num_groups           = Gp;
      gb->stats.num_groups      = Gp;
      gb->stats.strategy        = strategy;
      gb->stats.scratch_bytes   = static_cast<int64_t>(scratch.total());
      gb->stats.kernel_launches = launches;
      timer.read(gb->stats);
      return;
    }

    int64_t G          = 0;
    TableRef t{};
    uint32_t* map = nullptr;
    for (int attempt = 0;; ++attempt) {
      // ---- table
      t     = TableRef{};
      t.cap = cap;
      t.keys = static_cast<uint64_t*>(scratch.get((cap + 1) * plan.key.nwords * 8));
      t.rows = static_cast<uint32_t*>(scratch.get((cap + 1) * 4));
      for (int a = 0; a < nacc; ++a) t.acc[a] = scratch.get((cap + 1) * acc_bytes(plan.acc.kind[a]));
      t.special_used = reinterpret_cast<uint32_t*>(ctl + 28);
      t.status       = d_status;
      GBX_CUDA(cudaMemsetAsync(d_status, 0, 4, s));
      GBX_CUDA(launch_init_table(t, plan.acc, plan.key.nwords, call.dev.num_sms, s));
      launches += 1;
      timer.mark(2);
      const uint32_t max_probes = static_cast<uint32_t>(std::min<uint64_t>(cap, 1u << 12));
      if (strategy == GBX_STRATEGY_WARP) {
        GBX_CUDA(launch_agg_warp(plan, t, make_smem_layout(plan, s_warp), call.n, call.dev.num_sms, max_probes, s));
      } else if (strategy == GBX_STRATEGY_PRIVATIZED) {
        uint32_t S = static_cast<uint32_t>(std::min<uint64_t>(next_pow2(static_cast<uint64_t>(std::max(2.0 * est, 64.0))), s_max));
        if (skew_stream) S = stream_slots;
        const SmemLayout sl = make_smem_layout(plan, S);
        const int block = 512;
        int grid        = call.dev.num_sms * std::max<int>(1, std::min<int>(4, static_cast<int>((200 * 1024) / (sl.total + 1024))));
        int64_t max_grid = (call.n + block * 4 - 1) / (block * 4);
        grid             = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(grid, max_grid)));
        if (skew_stream) {
          // skewed keys: the streamed-tile kernel keeps the hot keys in shared
          // memory and sends the rare keys' rows to the global table
          // a short probe: a hot key was inserted early and sits near its home
          // slot; a rare key that misses goes to the global table
          GBX_CUDA(launch_agg_stream(plan, t, sl, call.n, call.dev.num_sms, std::min<uint32_t>(S, 8), max_probes, s));
        } else if (tiled_fits(sl, plan.nchan) && !arg_kinds) {
          // few groups: tiles grouped in shared memory before the table is touched
          GBX_CUDA(launch_agg_tiled(plan, t, sl, call.n, call.dev.num_sms, std::min<uint32_t>(S, 32), max_probes, s));
        } else {
          GBX_CUDA(launch_agg_privatized(plan, t, sl, call.n, block, grid, std::min<uint32_t>(S, 32), max_probes, s));
        }
      } else if (strategy == GBX_STRATEGY_BUCKETED) {
        // radix passes into bucket order, then tiles of the bucket-ordered
        // rows grouped in shared memory (gbx_tiled.cu)
        const PartBufs pb  = part_bufs();
        const PartBufs tmp = bucket_bits > 8 ? part_bufs() : pb;  // one pass writes `pb` only
        auto* rcounts      = static_cast<uint32_t*>(scratch.get(part_radix_count_bytes(call.n)));
        auto* roffsets     = static_cast<uint32_t*>(scratch.get(part_radix_count_bytes(call.n)));
        size_t rtemp_bytes = 0;
        GBX_CUDA(part_radix_temp_bytes(call.n, &rtemp_bytes));
        void* rtemp  = scratch.get(rtemp_bytes);
        auto* n_kept = static_cast<uint32_t*>(scratch.get(sizeof(uint32_t)));
        GBX_CUDA(launch_part_radix_hist0(plan, call.n, bucket_bits, rcounts, nullptr, s));
        GBX_CUDA(launch_part_radix(plan, call.n, bucket_bits, n_kept, pb, tmp, rcounts, roffsets, rtemp, rtemp_bytes,
                                   d_status, /*hist0_done=*/true, s));
        GBX_CUDA(launch_agg_tiled_part(plan, t, make_smem_layout(plan, bucket_slots), pb, n_kept, call.n,
                                       call.dev.num_sms, std::min<uint32_t>(bucket_slots, 32), max_probes, s));
        launches += 1 + 3 * ((bucket_bits + 7) / 8);  // first histogram, 3 per pass
      } else {
        GBX_CUDA(launch_agg_global(plan, t, call.n, max_probes, call.dev.num_sms, s));
      }
      launches += 1;
      timer.mark(3);
      // ---- compaction of occupied slots
      map = static_cast<uint32_t*>(scratch.get((cap + 1) * 4));
      GBX_CUDA(compact_occupied(t, plan.key.nwords, map, d_num_selected, call.dev.num_sms, s));
      launches += 1;
      timer.mark(4);
      GBX_CUDA(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      int32_t status;
      std::memcpy(&status, reinterpret_cast<char*>(h_ctl) + 26 * 8, 4);
      std::memcpy(&G, reinterpret_cast<char*>(h_ctl) + 27 * 8, 8);
      if (status & S_SPIN_LIMIT) fail(GBX_ERR_DEVICE, "a bounded device loop gave up (status 0x%x)", status);
      if (status & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");
      if (status & S_CHECK_FAILED) fail(GBX_ERR_DEVICE, "bucketed path: rows out of bucket order (status 0x%x)", status);
      if ((status & S_TABLE_FULL) == 0) break;
      // table too small for the groups present: grow and redo
      if (cap >= (1ULL << 31) || attempt >= 3) fail(GBX_ERR_DEVICE, "hash table overflow at capacity %llu", (unsigned long long)cap);
      gb->stats.retries++;
      scratch.release_all();
      ctl = static_cast<unsigned long long*>(scratch.get(kCtlWords * 8));
      GBX_CUDA(cudaMemsetAsync(ctl, 0, kCtlWords * 8, s));
      d_status       = reinterpret_cast<int32_t*>(ctl + 26);
      d_num_selected = reinterpret_cast<int64_t*>(ctl + 27);
      // grow 16x (an underestimate of a skewed key's tail is usually within
      // that), then to the bound of every row being a group
      const uint64_t bound = next_pow2(2 * static_cast<uint64_t>(call.n) + 2);
      cap = std::min<uint64_t>(attempt == 0 ? std::min<uint64_t>(cap * 16, bound) : std::max<uint64_t>(cap * 4, bound),
                               1ULL << 31);
      if (strategy == GBX_STRATEGY_WARP || strategy == GBX_STRATEGY_BUCKETED ||
          (strategy == GBX_STRATEGY_PRIVATIZED && !skew_stream))
        strategy = GBX_STRATEGY_GLOBAL;
      est = static_cast<double>(cap / 2);
    }
    gb->stats.strategy        = strategy;
    gb->stats.table_capacity  = static_cast<int64_t>(cap);
    if (strategy == GBX_STRATEGY_BUCKETED) {
      gb->stats.partition_bits = bucket_bits;
      gb->stats.bucket_slots   = static_cast<int32_t>(bucket_slots);
    }
    gb->stats.num_groups      = G;
    gb->stats.scratch_bytes   = static_cast<int64_t>(scratch.total());
    gb->stats.kernel_launches = launches + (G > 0 ? 1 : 0);  // + finalize
    res->num_groups           = G;

    // ---- outputs
    OutPlan op     = build_outputs(G);
    auto* d_nulls  = static_cast<unsigned long long*>(scratch.get((kMaxKeyCols + kMaxOut) * 8));
    GBX_CUDA(cudaMemsetAsync(d_nulls, 0, (kMaxKeyCols + kMaxOut) * 8, s));
    op.null_counts = d_nulls;
    GBX_CUDA(launch_finalize(plan, t, map, G, op, call.dev.num_sms, s));
    if (!sorted_outs.empty() && G > 0 && call.n > 0) {
      // ---- MEDIAN / QUANTILE / NUNIQUE / NTH_ELEMENT (gbx_sort.cu)
      GBX_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int32_t), s));
      double* d_q = nullptr;
      if (!h_quantiles.empty()) {
        d_q = static_cast<double*>(scratch.get(h_quantiles.size() * sizeof(double)));
        GBX_CUDA(cudaMemcpyAsync(d_q, h_quantiles.data(), h_quantiles.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
      }
      SortedKindsArgs sa{};
      sa.plan       = plan;
      sa.table      = t;
      sa.map        = map;
      sa.num_groups = G;
      sa.n          = call.n;
      sa.max_probes = static_cast<uint32_t>(std::min<uint64_t>(cap, 1u << 12));
      sa.scratch    = &scratch;
      sa.status     = d_status;
      sa.num_sms    = call.dev.num_sms;
      sa.stream     = s;
      for (size_t i = 0; i < sorted_outs.size(); ++i) {
        SortedOut so     = sorted_outs[i];
        so.quantiles_dev = d_q ? d_q + reinterpret_cast<uintptr_t>(so.quantiles_dev) : nullptr;
        so.null_count    = d_nulls + kMaxKeyCols + sorted_out_index[i];
        sa.outs.push_back(so);
      }
      // one sort of a channel's values serves all of its MEDIAN / QUANTILE /
      // NUNIQUE outputs: those first, channel by channel, NTH_ELEMENT last
      std::stable_sort(sa.outs.begin(), sa.outs.end(), [](const SortedOut& x, const SortedOut& y) {
        const bool nx = x.kind == GBX_AGG_NTH_ELEMENT, ny = y.kind == GBX_AGG_NTH_ELEMENT;
        if (nx != ny) return ny;
        return x.chan < y.chan;
      });
      int sort_launches = 0;
      sorted_kinds(sa, &sort_launches);
      gb->stats.kernel_launches += sort_launches;
    }
    timer.mark(5);
    std::vector<unsigned long long> h_nulls(kMaxKeyCols + kMaxOut, 0);
    int32_t sort_status = 0;
    GBX_CUDA(cudaMemcpyAsync(h_nulls.data(), d_nulls, h_nulls.size() * 8, cudaMemcpyDeviceToHost, s));
    if (!sorted_outs.empty())
      GBX_CUDA(cudaMemcpyAsync(&sort_status, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GBX_CUDA(cudaStreamSynchronize(s));
    if (sort_status & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");
    if (sort_status & (S_TABLE_FULL | S_SPIN_LIMIT))
      fail(GBX_ERR_DEVICE, "sorted kinds: a row's key was not found in the finished table (status 0x%x)", sort_status);
    for (int c = 0; c < nkeys; ++c)
      if (res->keys[c].null_mask) res->keys[c].view.null_count = static_cast<int64_t>(h_nulls[c]);
    {
      int o = 0;
      for (int q = 0; q < num_requests; ++q)
        for (int k = 0; k < requests[q].num_aggregations; ++k, ++o) {
          gbx_column& oc = res->requests[q].results[k];
          if (oc.null_mask) oc.view.null_count = static_cast<int64_t>(h_nulls[kMaxKeyCols + o]);
          if (requests[q].aggregations[k].kind == GBX_AGG_NTH_ELEMENT && oc.null_mask && oc.view.null_count == 0) {
            // group_nth_element.cu: no mask without nulls
            call.alloc.release(oc.null_mask, oc.mask_bytes);
            oc.null_mask      = nullptr;
            oc.mask_bytes     = 0;
            oc.view.null_mask = nullptr;
          }
        }
    }
    timer.read(gb->stats);
    // scratch is released stream-ordered by ~Scratch
  });
  if (st == GBX_OK && pack_args) {
    if (res) gbx_result_release(res);
    res = nullptr;
    st  = guarded([&] {
      aggregate_with_packed_args(gb, gb->keys.empty() ? 0 : gb->keys[0].size, requests, num_requests, stream, mr, &res);
    });
  }
  if (st != GBX_OK) {
    if (res) gbx_result_release(res);
    return st;
  }
  *out = res;
  return GBX_OK;
}

}  // extern "C"

// ============================================= groupby without allocation

namespace gbx {
cudaError_t noalloc_scratch(void** ptr, size_t* bytes);  // gbx_noalloc.cu
}

extern "C" int gbx_groupby_aggregate_noalloc(gbx_groupby* gb,
                                             const gbx_request* requests,
                                             int32_t num_requests,
                                             void* stream,
                                             gbx_column* out_keys,
                                             gbx_column* out_results,
                                             int64_t capacity,
                                             int64_t* num_groups)
{
  return guarded([&] {
    GBX_EXPECTS(gb != nullptr && num_groups != nullptr, "null argument");
    *num_groups = 0;
    validate(gb, requests, num_requests);
    if (gb->keys_are_sorted)
      fail(GBX_ERR_UNSUPPORTED, "keys declared sorted group by runs, which need scratch in proportion to the rows; "
                                "use gbx_groupby_aggregate");
    if (keys_need_representatives(gb->keys, gb->null_policy))
      fail(GBX_ERR_UNSUPPORTED, "STRING keys and keys beyond 128 packed bits need scratch in proportion to the rows; "
                                "use gbx_groupby_aggregate");
    for (int q = 0; q < num_requests; ++q)
      for (int k = 0; k < requests[q].num_aggregations; ++k)
        if (is_sort_kind(requests[q].aggregations[k].kind))
          fail(GBX_ERR_UNSUPPORTED,
               "MEDIAN / QUANTILE / NUNIQUE / NTH_ELEMENT sort every row's value and need scratch in proportion "
               "to the rows; use gbx_groupby_aggregate");
    const int nkeys = static_cast<int>(gb->keys.size());
    int nout        = 0;
    for (int q = 0; q < num_requests; ++q) nout += requests[q].num_aggregations;
    GBX_EXPECTS(nkeys == 0 || out_keys != nullptr, "out_keys is null");
    GBX_EXPECTS(nout == 0 || out_results != nullptr, "out_results is null");
    GBX_EXPECTS(capacity >= 0, "negative capacity");
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    DeviceInfo dev  = current_device();
    const int64_t n = gb->keys.empty() ? 0 : gb->keys[0].size;

    // ---- the fixed scratch array of this device (and, on the first call in
    //      this context, the array and the path's kernels loaded there)
    void* base        = nullptr;
    size_t base_bytes = 0;
    GBX_CUDA(noalloc_scratch(&base, &base_bytes));
    size_t off = 0;
    auto carve = [&](size_t bytes) -> void* {
      off       = (off + 255) & ~size_t(255);
      void* p   = static_cast<char*>(base) + off;
      off      += bytes;
      if (off > base_bytes)
        fail(GBX_ERR_LOGIC,
             "the aggregations' per-group state exceeds the %u-byte scratch of the no-allocation groupby; "
             "use gbx_groupby_aggregate",
             GBX_NOALLOC_SCRATCH_BYTES);
      return p;
    };
    constexpr int kCtlWords = 32;
    auto* ctl               = static_cast<unsigned long long*>(carve(kCtlWords * 8));
    auto* d_nulls           = static_cast<unsigned long long*>(carve((kMaxKeyCols + kMaxOut) * 8));

    // ---- distinct value columns -> channels
    std::vector<int> req_chan;
    std::vector<const gbx_column_view*> chan_cols = collect_channels(requests, num_requests, req_chan);
    if (nout > kMaxOut) fail(GBX_ERR_UNSUPPORTED, "more than %d results in one call", kMaxOut);

    // ---- null counts of masks with an unknown count
    std::vector<int64_t> key_nulls(nkeys, 0), chan_nulls(chan_cols.size(), 0);
    MaskSpans ms{};
    std::vector<std::pair<int, int>> span_owner;
    for (int c = 0; c < nkeys; ++c) {
      key_nulls[c] = exact_null_count_or_neg(gb->keys[c]);
      if (key_nulls[c] < 0) {
        ms.span[ms.n++] = MaskSpan{gb->keys[c].null_mask, gb->keys[c].offset, gb->keys[c].size};
        span_owner.push_back({0, c});
      }
    }
    for (size_t c = 0; c < chan_cols.size(); ++c) {
      chan_nulls[c] = exact_null_count_or_neg(*chan_cols[c]);
      if (chan_nulls[c] < 0) {
        ms.span[ms.n++] = MaskSpan{chan_cols[c]->null_mask, chan_cols[c]->offset, chan_cols[c]->size};
        span_owner.push_back({1, static_cast<int>(c)});
      }
    }
    unsigned long long h_ctl[kCtlWords];
    GBX_CUDA(cudaMemsetAsync(ctl, 0, kCtlWords * 8, s));
    if (ms.n > 0 && n > 0) {
      GBX_CUDA(launch_count_valid(ms, ctl + 2, dev.num_sms, s));
      GBX_CUDA(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      for (size_t i = 0; i < span_owner.size(); ++i) {
        int64_t nulls = ms.span[i].size - static_cast<int64_t>(h_ctl[2 + i]);
        if (span_owner[i].first == 0) key_nulls[span_owner[i].second] = nulls;
        else chan_nulls[span_owner[i].second] = nulls;
      }
    } else {
      for (int c = 0; c < nkeys; ++c) key_nulls[c] = std::max<int64_t>(key_nulls[c], 0);
      for (auto& v : chan_nulls) v = std::max<int64_t>(v, 0);
    }

    // ---- plan: packed keys and one accumulator set per channel
    bool key_ok = true;
    Plan plan{};
    plan.key = make_key_plan(gb->keys.data(), nkeys, gb->null_policy, key_nulls, key_ok);
    if (!key_ok)
      fail(GBX_ERR_UNSUPPORTED, "key columns need more than 128 packed bits; wider composite keys are not supported");
    fill_channels(plan, chan_cols, chan_nulls, requests, num_requests, req_chan);
    const int nacc = plan.acc.nacc;

    // ---- fixed-capacity global table carved from the scratch array
    const uint64_t cap = 2ull * GBX_NOALLOC_MAX_GROUPS;
    TableRef t{};
    t.cap          = cap;
    t.keys         = static_cast<uint64_t*>(carve((cap + 1) * plan.key.nwords * 8));
    t.rows         = static_cast<uint32_t*>(carve((cap + 1) * 4));
    for (int a = 0; a < nacc; ++a) t.acc[a] = carve((cap + 1) * acc_bytes(plan.acc.kind[a]));
    t.special_used = reinterpret_cast<uint32_t*>(ctl + 28);
    t.status       = reinterpret_cast<int32_t*>(ctl + 26);
    auto* map      = static_cast<uint32_t*>(carve((cap + 1) * 4));
    auto* d_num_selected = reinterpret_cast<int64_t*>(ctl + 27);

    int64_t G = 0;
    if (n > 0) {
      GBX_CUDA(launch_init_table(t, plan.acc, plan.key.nwords, dev.num_sms, s));
      GBX_CUDA(launch_agg_global(plan, t, n, static_cast<uint32_t>(std::min<uint64_t>(cap, 1u << 12)), dev.num_sms, s));
      GBX_CUDA(compact_occupied(t, plan.key.nwords, map, d_num_selected, dev.num_sms, s));
      GBX_CUDA(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      int32_t status;
      std::memcpy(&status, reinterpret_cast<char*>(h_ctl) + 26 * 8, 4);
      std::memcpy(&G, reinterpret_cast<char*>(h_ctl) + 27 * 8, 8);
      if (status & S_SPIN_LIMIT) fail(GBX_ERR_DEVICE, "a bounded device loop gave up (status 0x%x)", status);
      if (status & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");
      if ((status & S_TABLE_FULL) || G > GBX_NOALLOC_MAX_GROUPS)
        fail(GBX_ERR_LOGIC, "the input has more than %d groups, the limit of the no-allocation groupby",
             GBX_NOALLOC_MAX_GROUPS);
    }
    GBX_EXPECTS(G <= capacity, "the input has %lld groups but the outputs hold %lld rows", (long long)G,
                (long long)capacity);

    // ---- describe the caller's output columns
    OutPlan op{};
    auto describe = [&](gbx_column& c, int32_t type_id, int32_t scale, bool with_mask) {
      GBX_EXPECTS(G == 0 || c.data != nullptr, "an output column has no data buffer");
      GBX_EXPECTS(!with_mask || G == 0 || c.null_mask != nullptr, "a nullable output column has no null_mask buffer");
      c.view            = gbx_column_view{};
      c.view.type_id    = type_id;
      c.view.scale      = scale;
      c.view.size       = G;
      c.view.data       = c.data;
      c.view.null_mask  = with_mask ? c.null_mask : nullptr;
      c.view.null_count = 0;
    };
    for (int c = 0; c < nkeys; ++c) {
      const gbx_column_view& kcv = gb->keys[c];
      bool with_mask             = plan.key.cols[c].null_bit != 0;
      describe(out_keys[c], kcv.type_id, kcv.scale, with_mask);
      if (kcv.type_id == GBX_TYPE_DICTIONARY32) {
        out_keys[c].view.index_type_id = kcv.index_type_id ? kcv.index_type_id : GBX_TYPE_INT32;
        out_keys[c].view.dict_keys     = kcv.dict_keys;
      }
      op.key_data[c] = out_keys[c].data;
      op.key_mask[c] = with_mask ? out_keys[c].null_mask : nullptr;
    }
    int o = 0;
    for (int q = 0; q < num_requests; ++q) {
      const gbx_request& r = requests[q];
      int32_t vt           = value_type(r.values);
      for (int k = 0; k < r.num_aggregations; ++k, ++o) {
        int32_t kind   = r.aggregations[k].kind;
        int32_t tt     = target_type(vt, kind);
        bool with_mask = (kind == GBX_AGG_COUNT_VALID || kind == GBX_AGG_COUNT_ALL)
                           ? false
                           : (chan_nulls[req_chan[q]] != 0 || kind == GBX_AGG_VARIANCE || kind == GBX_AGG_STD);
        int32_t scale  = is_decimal(tt) ? (r.values.type_id == GBX_TYPE_DICTIONARY32 ? r.values.dict_keys->scale
                                                                                     : r.values.scale)
                                        : 0;
        describe(out_results[o], tt, scale, with_mask);
        OutCol& oc   = op.out[op.nout++];
        oc.data      = out_results[o].data;
        oc.mask      = with_mask ? out_results[o].null_mask : nullptr;
        oc.kind      = kind;
        oc.ddof      = r.aggregations[k].ddof;
        oc.chan      = static_cast<int8_t>(req_chan[q]);
        oc.out_ptype = phys_of(tt);
        oc.out_width = static_cast<int8_t>(type_width(tt));
      }
    }
    if (G > 0) {
      GBX_CUDA(cudaMemsetAsync(d_nulls, 0, (kMaxKeyCols + kMaxOut) * 8, s));
      op.null_counts = d_nulls;
      GBX_CUDA(launch_finalize(plan, t, map, G, op, dev.num_sms, s));
      unsigned long long h_nulls[kMaxKeyCols + kMaxOut];
      GBX_CUDA(cudaMemcpyAsync(h_nulls, d_nulls, sizeof(h_nulls), cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      for (int c = 0; c < nkeys; ++c)
        if (op.key_mask[c]) out_keys[c].view.null_count = static_cast<int64_t>(h_nulls[c]);
      for (int i = 0; i < op.nout; ++i)
        if (op.out[i].mask) out_results[i].view.null_count = static_cast<int64_t>(h_nulls[kMaxKeyCols + i]);
    }
    *num_groups = G;
  });
}
