// gbx_sort.cu -- the kinds libcudf computes on its sort-based groupby
// (MEDIAN, QUANTILE, NUNIQUE, NTH_ELEMENT), over the groups of the hash table.
//
// The reference sorts the keys, labels each row with its group and sorts a
// request's values within their groups (groupby/sort/sort_helper.cu:251-272,
// groupby/sort/aggregate.cpp:323-406, group_quantiles.cu, group_nunique.cu,
// group_nth_element.cu).  Here the groups are already known from the hash
// table: every row's label is the output row of its key (a probe of the
// finished table), and only the (label, value) records of a request are put
// in order, by an LSD radix sort of libgbx's own: 8-bit digits, each pass a
// stable counting sort over 4,096-record tiles (tile histograms, one
// exclusive scan over (digit, tile), ranks by warp-aggregated counts in tile
// order).
//
// Two record formats.  Packed, one 64-bit word, whenever it fits:
//   values: label << (vbits + 1) | null << vbits | (order key - min key)
//   rows:   label << rbits | row                     (NTH_ELEMENT)
// where a row whose key is excluded takes label G (after every group), vbits
// covers the value range seen (a reduction over the rows first) and rbits the
// row count; only the bits in use are sorted (rows: the label bits alone, so a
// group's rows stay in row order).  Split, when the value range is too wide
// (float64, or values with -0.0 that a float32's key cannot keep):
//   hi (32 bits) = label << 1 | null (excluded rows: 1 << (lbits + 1)),
//   lo (64 bits) = the order key (a float32's own bits above its 32-bit key).
// After the sort each group's records are contiguous: valid values first, in
// ascending order, then the nulls.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "gbx_host.hpp"
#include "gbx_kernels.hpp"
#include "gbx_scan.hpp"
#include "gbx_sort.hpp"
#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kSortBlock    = 256;
constexpr int kSortWarps    = kSortBlock / 32;
constexpr int kSortPerWarp  = 512;
constexpr int kSortTile     = kSortWarps * kSortPerWarp;
constexpr uint32_t kNoLabel = 0xffffffffu;

// ------------------------------------------------------------ order keys

// An unsigned key that orders the values of physical type pt as the
// reference's sort does: equal for equal values (-0.0 and +0.0 one key, every
// NaN one key), NaN after every number (the relational comparator of
// table/experimental/row_operators.cuh).  A float's key is 32 bits wide.
__device__ __forceinline__ uint64_t order_key(uint64_t b, int pt)
{
  switch (pt) {
    case P_I8: return static_cast<uint8_t>(static_cast<uint8_t>(b) ^ 0x80u);
    case P_I16: return static_cast<uint16_t>(static_cast<uint16_t>(b) ^ 0x8000u);
    case P_I32: return static_cast<uint32_t>(static_cast<uint32_t>(b) ^ 0x80000000u);
    case P_I64: return b ^ 0x8000000000000000ULL;
    case P_F32: {
      uint32_t u    = static_cast<uint32_t>(b);
      const float f = __uint_as_float(u);
      if (f != f) u = 0x7fc00000u;
      else if (f == 0.0f) u = 0;
      return (u & 0x80000000u) ? static_cast<uint32_t>(~u) : (u | 0x80000000u);
    }
    case P_F64: {
      uint64_t u     = b;
      const double d = __longlong_as_double(static_cast<long long>(u));
      if (d != d) u = 0x7ff8000000000000ULL;
      else if (d == 0.0) u = 0;
      return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
    }
    case P_BOOL: return b != 0;
    default: return b;  // unsigned
  }
}

// The value bits of an order key (a zero comes back as +0.0, a NaN as the
// canonical quiet NaN).
__device__ __forceinline__ uint64_t key_decode(uint64_t k, int pt)
{
  switch (pt) {
    case P_I8: return static_cast<uint8_t>(static_cast<uint8_t>(k) ^ 0x80u);
    case P_I16: return static_cast<uint16_t>(static_cast<uint16_t>(k) ^ 0x8000u);
    case P_I32: return static_cast<uint32_t>(static_cast<uint32_t>(k) ^ 0x80000000u);
    case P_I64: return k ^ 0x8000000000000000ULL;
    case P_F32: {
      const uint32_t u = static_cast<uint32_t>(k);
      return (u & 0x80000000u) ? (u & 0x7fffffffu) : static_cast<uint32_t>(~u);
    }
    case P_F64: return (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    default: return k;
  }
}

// True for a float value of -0.0 (whose key does not keep the sign).
__device__ __forceinline__ bool is_neg_zero(uint64_t b, int pt)
{
  if (pt == P_F32) return static_cast<uint32_t>(b) == 0x80000000u;
  if (pt == P_F64) return b == 0x8000000000000000ULL;
  return false;
}

// --------------------------------------------------------------- formats

// How a sorted record reads back.  Packed: `shift` = the label's bit offset
// (vbits + 1, or rbits), `nullbit` = 1 << vbits (0 for rows), `vmask` the
// value / row bits, `kmin` the order key subtracted.  Split: lo is the order
// key (float32: the row's bits above it), hi the label word.
struct Fmt {
  bool split;
  int shift;
  uint64_t nullbit;
  uint64_t vmask;
  uint64_t kmin;
};

template <bool kSplit>
__device__ __forceinline__ uint64_t rec_value(const Fmt& f, uint64_t lo, int pt)
{
  if constexpr (kSplit) return pt == P_F32 ? (lo >> 32) : key_decode(lo, pt);
  else return key_decode((lo & f.vmask) + f.kmin, pt);
}

// ------------------------------------------------------------- labels

// inv[map[g]] = g: each occupied slot's output row.
__global__ void k_slot_rows(const uint32_t* __restrict__ map, int64_t G, uint32_t* __restrict__ inv)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x)
    inv[map[g]] = static_cast<uint32_t>(g);
}

// labels[r] = the output row of row r's group (kNoLabel for a row whose key
// is excluded); every key is in the table, so the probe only finds.
template <int NW>
__global__ void k_row_labels(const __grid_constant__ Plan plan, const __grid_constant__ TableRef t, int64_t n,
                             const uint32_t* __restrict__ inv, uint32_t max_probes, uint32_t* __restrict__ labels)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t k[NW];
    uint32_t label = kNoLabel;
    if (pack_key<NW>(plan.key, r, k)) {
      const int64_t s = global_slot<NW>(t, k, max_probes);
      if (s >= 0) label = inv[s];
    }
    labels[r] = label;
  }
}

// --------------------------------------------------------------- records

// The smallest and largest order key of the channel's valid values in
// labelled rows, whether any is -0.0, whether any exists.
struct Range {
  unsigned long long kmin, kmax;
  unsigned int neg_zero, any;
};

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int o)
{
  return __shfl_xor_sync(0xffffffffu, v, o);
}

__global__ void k_value_range(const __grid_constant__ Channel ch, int64_t n, const uint32_t* __restrict__ labels,
                              Range* out, int32_t* status)
{
  unsigned long long lo = ~0ULL, hi = 0;
  bool neg0 = false, any = false;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t n_up   = (n + 31) & ~int64_t(31);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_up; r += stride) {
    if (r < n && labels[r] != kNoLabel && bit_valid(ch.mask, r + ch.offset)) {
      bool ok;
      const uint64_t b = value_bits(ch, r, ok);
      if (ok) {
        const uint64_t k = order_key(b, ch.ptype);
        lo               = k < lo ? k : lo;
        hi               = k > hi ? k : hi;
        neg0             = neg0 || is_neg_zero(b, ch.ptype);
        any              = true;
      } else {
        atomicOr(status, S_BAD_INDEX);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long l2 = shfl_xor_u64(lo, o), h2 = shfl_xor_u64(hi, o);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  neg0 = __any_sync(0xffffffffu, neg0);
  any  = __any_sync(0xffffffffu, any);
  if ((threadIdx.x & 31) == 0 && any) {
    atomicMin(&out->kmin, lo);
    atomicMax(&out->kmax, hi);
    atomicOr(&out->any, 1u);
    if (neg0) atomicOr(&out->neg_zero, 1u);
  }
}

// Packed records.  Values: label << (vbits + 1) | null << vbits | (key - kmin)
// (skip_nulls: null values take label G too).  Rows: label << rbits | row.
__global__ void k_records_packed(const __grid_constant__ Channel ch, int64_t n, const uint32_t* __restrict__ labels,
                                 bool rows_mode, bool skip_nulls, uint32_t G, int vbits, uint64_t kmin,
                                 uint64_t* __restrict__ rec, int32_t* status)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t label = labels[r];
    if (label == kNoLabel) label = G;
    uint64_t b = 0;
    bool valid = false;
    if (label != G && bit_valid(ch.mask, r + ch.offset)) {
      bool ok;
      b     = value_bits(ch, r, ok);
      valid = ok;
      if (!ok) atomicOr(status, S_BAD_INDEX);
    }
    if (skip_nulls && !valid) label = G;
    uint64_t w;
    if (rows_mode) {
      w = (static_cast<uint64_t>(label) << vbits) | static_cast<uint64_t>(r);
    } else {
      const uint64_t v = valid ? order_key(b, ch.ptype) - kmin : 0;
      w = (static_cast<uint64_t>(label) << (vbits + 1)) | ((label != G && !valid) ? (1ULL << vbits) : 0) | v;
    }
    rec[r] = w;
  }
}

// Split records: hi = label << 1 | null (excluded: skip_hi), lo = order key
// (a float32's own bits above its 32-bit key, not sorted on, so the value
// read back is the row's: -0.0 and NaN payloads kept).
__global__ void k_records_split(const __grid_constant__ Channel ch, int64_t n, const uint32_t* __restrict__ labels,
                                uint32_t skip_hi, uint64_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                int32_t* status)
{
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t label = labels[r];
    uint64_t b           = 0;
    bool valid           = false;
    if (label != kNoLabel && bit_valid(ch.mask, r + ch.offset)) {
      bool ok;
      b     = value_bits(ch, r, ok);
      valid = ok;
      if (!ok) atomicOr(status, S_BAD_INDEX);
    }
    hi[r] = label == kNoLabel ? skip_hi : ((label << 1) | (valid ? 0u : 1u));
    uint64_t l = 0;
    if (valid) {
      l = order_key(b, ch.ptype);
      if (ch.ptype == P_F32) l |= b << 32;
    }
    lo[r] = l;
  }
}

// ------------------------------------------------------------- radix sort

// Digit of a record at bit `shift`: of lo for shift < 64, else of hi at
// shift - 64 (split records only).
template <bool kSplit>
__device__ __forceinline__ uint32_t digit_at(uint64_t lo, uint32_t hi, int shift)
{
  if constexpr (kSplit)
    return shift < 64 ? static_cast<uint32_t>(lo >> shift) & 0xffu : (hi >> (shift - 64)) & 0xffu;
  else return static_cast<uint32_t>(lo >> shift) & 0xffu;
}

// counts[d * ntiles + tile] = records of the tile with digit d.
template <bool kSplit>
__global__ void __launch_bounds__(kSortBlock) k_sort_hist(const uint64_t* __restrict__ lo,
                                                          const uint32_t* __restrict__ hi, int64_t n, int shift,
                                                          int ntiles, uint32_t* __restrict__ counts)
{
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += kSortBlock) h[i] = 0;
  __syncthreads();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
  const bool use_hi  = kSplit && shift >= 64;
  for (int i = threadIdx.x; i < kSortTile; i += kSortBlock) {
    const int64_t r = base + i;
    if (r < n) atomicAdd(&h[digit_at<kSplit>(use_hi ? 0 : lo[r], use_hi ? hi[r] : 0, shift)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += kSortBlock) counts[static_cast<size_t>(i) * ntiles + blockIdx.x] = h[i];
}

// Stable scatter of one tile: the record at tile position (warp, batch,
// lane) -- row order -- goes to offsets[d * ntiles + tile] plus its rank
// among the tile's records of digit d.  Each lane keeps its 16 records and
// their ranks within the warp in registers (the ranking runs once); the tile
// is then laid out in shared memory in digit order and written out digit run
// by digit run with consecutive threads on consecutive rows, so that a warp's
// stores cover whole sectors.  The pass mostly waits on its tile's loads, so
// the packed-record form is held to three CTAs an SM (80 registers, a few
// spilled): the extra resident warps hide more of that wait than the spills
// cost.
template <bool kSplit>
__global__ void __launch_bounds__(kSortBlock, kSplit ? 2 : 3) k_sort_scatter(const uint64_t* __restrict__ lo_in,
                                                             const uint32_t* __restrict__ hi_in, int64_t n,
                                                             int shift, int ntiles,
                                                             const uint32_t* __restrict__ offsets,
                                                             uint64_t* __restrict__ lo_out,
                                                             uint32_t* __restrict__ hi_out)
{
  constexpr int kBatches = kSortPerWarp / 32;
  static_assert(kSortBlock == 256, "one thread per digit");
  __shared__ uint32_t cnt[kSortWarps][256];
  __shared__ uint32_t dstart[256];   // the digit's first position in the tile
  __shared__ uint32_t gstart[256];   // the digit run's first output row
  __shared__ uint32_t wsum[kSortWarps];
  // the staged tile (dynamic shared memory: scatter_smem_bytes)
  extern __shared__ __align__(16) unsigned char sort_stage[];
  uint64_t* stage_lo = reinterpret_cast<uint64_t*>(sort_stage);
  uint32_t* stage_hi = reinterpret_cast<uint32_t*>(sort_stage + kSortTile * sizeof(uint64_t));
  const int lane      = threadIdx.x & 31;
  const int warp      = threadIdx.x >> 5;
  const uint32_t lt   = (1u << lane) - 1u;
  const int64_t tile0 = static_cast<int64_t>(blockIdx.x) * kSortTile;
  const int64_t base  = tile0 + warp * kSortPerWarp;
  const int tile_n    = static_cast<int>(n - tile0 < kSortTile ? n - tile0 : kSortTile);
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortBlock) (&cnt[0][0])[i] = 0;
  uint64_t l[kBatches];
  uint32_t h[kBatches];
  uint32_t rank[kBatches];
#pragma unroll
  for (int j = 0; j < kBatches; ++j) {
    const int64_t r = base + j * 32 + lane;
    l[j]            = r < n ? lo_in[r] : 0;
    h[j]            = 0;
    if constexpr (kSplit) h[j] = r < n ? hi_in[r] : 0;
  }
  __syncthreads();
  // ranks within the warp, digit by digit in row order
#pragma unroll
  for (int j = 0; j < kBatches; ++j) {
    const int64_t r     = base + j * 32 + lane;
    const uint32_t act  = __ballot_sync(0xffffffffu, r < n);
    const uint32_t d    = digit_at<kSplit>(l[j], h[j], shift);
    const uint32_t pe   = digit_peers(d, 8, act);
    const bool mine     = (act >> lane) & 1u;
    const uint32_t prev = mine ? cnt[warp][d] : 0u;
    rank[j]             = prev + static_cast<uint32_t>(__popc(pe & lt));
    __syncwarp();
    if (mine && (pe & lt) == 0) cnt[warp][d] = prev + static_cast<uint32_t>(__popc(pe));
    __syncwarp();
  }
  __syncthreads();
  // thread d: the warps' bases within digit d, the digit's tile count, then
  // an exclusive scan of the counts over the digits (kSortBlock == 256)
  {
    const int d   = threadIdx.x;
    uint32_t tot  = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = cnt[w][d];
      cnt[w][d]        = tot;
      tot += c;
    }
    uint32_t x = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    dstart[d] = before + x - tot;
    gstart[d] = offsets[static_cast<size_t>(d) * ntiles + blockIdx.x];
  }
  __syncthreads();
  // the tile in digit order in shared memory
#pragma unroll
  for (int j = 0; j < kBatches; ++j) {
    const int64_t r = base + j * 32 + lane;
    if (r < n) {
      const uint32_t d  = digit_at<kSplit>(l[j], h[j], shift);
      const uint32_t at = dstart[d] + cnt[warp][d] + rank[j];
      stage_lo[at]      = l[j];
      if constexpr (kSplit) stage_hi[at] = h[j];
    }
  }
  __syncthreads();
  // digit runs out: position i of the tile is record i - dstart[d] of digit d
  for (int i = threadIdx.x; i < tile_n; i += kSortBlock) {
    const uint64_t v  = stage_lo[i];
    uint32_t hv       = 0;
    if constexpr (kSplit) hv = stage_hi[i];
    const uint32_t d  = digit_at<kSplit>(v, hv, shift);
    const uint32_t at = gstart[d] + static_cast<uint32_t>(i) - dstart[d];
    lo_out[at]        = v;
    if constexpr (kSplit) hi_out[at] = hv;
  }
}

// Dynamic shared memory of k_sort_scatter: the staged tile.
constexpr size_t scatter_smem_bytes(bool split)
{
  return kSortTile * sizeof(uint64_t) + (split ? kSortTile * sizeof(uint32_t) : 0);
}

// --------------------------------------------------------------- bounds

// First index of sorted `a` (n values) whose value is >= v.
template <class T>
__device__ __forceinline__ int64_t lower_bound(const T* a, int64_t n, T v)
{
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// bounds[3 g .. 3 g + 2] = group g's first record, first null record, end.
template <bool kSplit>
__global__ void k_group_bounds(const uint64_t* __restrict__ lo, const uint32_t* __restrict__ hi, int64_t n,
                               int64_t G, const Fmt f, int64_t* __restrict__ bounds)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if constexpr (kSplit) {
      const uint32_t key = static_cast<uint32_t>(g) << 1;
      bounds[3 * g]      = lower_bound<uint32_t>(hi, n, key);
      bounds[3 * g + 1]  = lower_bound<uint32_t>(hi, n, key | 1u);
      bounds[3 * g + 2]  = lower_bound<uint32_t>(hi, n, key + 2u);
    } else {
      const uint64_t key = static_cast<uint64_t>(g) << f.shift;
      const int64_t end  = lower_bound<uint64_t>(lo, n, static_cast<uint64_t>(g + 1) << f.shift);
      bounds[3 * g]      = lower_bound<uint64_t>(lo, n, key);
      bounds[3 * g + 1]  = f.nullbit ? lower_bound<uint64_t>(lo, n, key | f.nullbit) : end;
      bounds[3 * g + 2]  = end;
    }
  }
}

// --------------------------------------------------------------- results

// interpolate::midpoint of two values as double (quantiles_util.hpp:56-72):
// the int64 overload keeps the halves apart so that the sum cannot overflow
__device__ __forceinline__ double midpoint_of(uint64_t a, uint64_t b, int pt)
{
  if (pt == P_I64) {
    const int64_t x = static_cast<int64_t>(a), y = static_cast<int64_t>(b);
    const int64_t half = x / 2 + y / 2;
    const int64_t rest = x % 2 + y % 2;
    return __dadd_rn(static_cast<double>(half), static_cast<double>(rest) * 0.5);
  }
  return __dadd_rn(__dmul_rn(as_f64(a, pt), 0.5), __dmul_rn(as_f64(b, pt), 0.5));
}

// QUANTILE (MEDIAN: {0.5}, LINEAR) of each group's valid values, with the
// reference's quantile_index and interpolations (quantiles_util.hpp:92-190),
// result row g * nq + j for group g and quantile j.
template <bool kSplit>
__global__ void k_quantiles(const uint64_t* __restrict__ lo, const int64_t* __restrict__ bounds, int64_t G,
                            const Fmt f, int pt, const double* __restrict__ qs, int nq, int interp,
                            double* __restrict__ out, uint32_t* __restrict__ mask, unsigned long long* null_count)
{
  const int lane      = threadIdx.x & 31;
  const int64_t total = G * nq;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31); base < total;
       base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i   = base + lane;
    const bool active = i < total;
    bool valid        = false;
    if (active) {
      const int64_t g     = i / nq;
      const int64_t start = bounds[3 * g];
      const int64_t count = bounds[3 * g + 1] - start;
      double v            = 0.0;
      valid               = count > 0;
      if (valid) {
        // plain double operations, each rounded on its own (no fused
        // multiply-add), in the reference's order
        const double q    = fmin(fmax(qs[i % nq], 0.0), 1.0);
        const double val  = __dmul_rn(q, static_cast<double>(count - 1));
        const int64_t lwr = static_cast<int64_t>(floor(val));
        const int64_t hgr = static_cast<int64_t>(ceil(val));
        const int64_t nst = static_cast<int64_t>(nearbyint(val));
        const double frac = val - static_cast<double>(lwr);
        const uint64_t a  = rec_value<kSplit>(f, lo[start + lwr], pt);
        const uint64_t b  = rec_value<kSplit>(f, lo[start + hgr], pt);
        switch (interp) {
          case GBX_INTERP_LOWER: v = as_f64(a, pt); break;
          case GBX_INTERP_HIGHER: v = as_f64(b, pt); break;
          case GBX_INTERP_NEAREST: v = as_f64(rec_value<kSplit>(f, lo[start + nst], pt), pt); break;
          case GBX_INTERP_MIDPOINT: v = midpoint_of(a, b, pt); break;
          default: v = __dadd_rn(__dmul_rn(1.0 - frac, as_f64(a, pt)), __dmul_rn(frac, as_f64(b, pt))); break;
        }
      }
      out[i] = v;
    }
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    const uint32_t bal = __ballot_sync(0xffffffffu, active && valid);
    if (lane == 0 && act != 0) {
      // base stays a multiple of 32 (the stride is), so word base / 32 is
      // this warp's alone
      mask[base >> 5] = bal;
      const uint32_t nulls = __popc(act & ~bal);
      if (nulls) atomicAdd(null_count, static_cast<unsigned long long>(nulls));
    }
  }
}

// first[i] = 1 when record i holds a (group, value) pair not seen at i - 1;
// only the order key's bits (`key_mask`) of a split record's lo are compared.
template <bool kSplit>
__global__ void k_distinct_flags(const uint64_t* __restrict__ lo, const uint32_t* __restrict__ hi, int64_t n,
                                 uint64_t key_mask, uint32_t* __restrict__ first)
{
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    bool f = i == 0;
    if (!f) {
      if constexpr (kSplit) f = hi[i] != hi[i - 1] || ((lo[i] ^ lo[i - 1]) & key_mask) != 0;
      else f = lo[i] != lo[i - 1];
    }
    first[i] = f ? 1u : 0u;
  }
}

// NUNIQUE: the group's distinct valid values, plus one for its nulls under
// INCLUDE (group_nunique.cu:63-72), from the exclusive scan of the flags.
__global__ void k_nunique(const uint32_t* __restrict__ scanned, const int64_t* __restrict__ bounds, int64_t G,
                          bool include_nulls, int32_t* __restrict__ out)
{
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = bounds[3 * g], vend = bounds[3 * g + 1], e = bounds[3 * g + 2];
    int32_t c       = static_cast<int32_t>(scanned[vend] - scanned[s]);
    if (include_nulls && e > vend) ++c;
    out[g] = c;
  }
}

// NTH_ELEMENT: the n-th record of each group in row order (negative n from
// the end); null when out of range or when that row's value is null
// (group_nth_element.cu).  Records are packed rows (row = rec & vmask).
__global__ void k_nth_element(const __grid_constant__ Channel ch, const uint64_t* __restrict__ rec,
                              const int64_t* __restrict__ bounds, int64_t G, uint64_t row_mask, int64_t nth,
                              int width, void* __restrict__ out, uint32_t* __restrict__ mask,
                              unsigned long long* null_count, int32_t* status)
{
  const int lane = threadIdx.x & 31;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31); base < G;
       base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t g   = base + lane;
    const bool active = g < G;
    bool valid        = false;
    if (active) {
      uint64_t v        = 0;
      const int64_t s   = bounds[3 * g];
      const int64_t len = bounds[3 * g + 2] - s;
      const int64_t idx = nth >= 0 ? nth : len + nth;
      if (idx >= 0 && idx < len) {
        const int64_t row = static_cast<int64_t>(rec[s + idx] & row_mask);
        if (bit_valid(ch.mask, row + ch.offset)) {
          bool ok;
          v     = value_bits(ch, row, ok);
          valid = ok;
          if (!ok) atomicOr(status, S_BAD_INDEX);
        }
      }
      store_bits(out, g, width, valid ? v : 0);
    }
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    const uint32_t bal = __ballot_sync(0xffffffffu, active && valid);
    if (lane == 0 && act != 0) {
      mask[base >> 5] = bal;
      const uint32_t nulls = __popc(act & ~bal);
      if (nulls) atomicAdd(null_count, static_cast<unsigned long long>(nulls));
    }
  }
}

int grid_of(int64_t work, int num_sms)
{
  const int64_t b = (work + 255) / 256;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(num_sms) * 8)));
}

int bits_for(uint64_t v)
{
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

}  // namespace

void sorted_kinds(const SortedKindsArgs& a, int* launches)
{
  const int64_t n = a.n;
  const int64_t G = a.num_groups;
  cudaStream_t s  = a.stream;
  if (a.outs.empty() || n == 0 || G == 0) return;
  if (G >= (int64_t(1) << 30)) fail(GBX_ERR_UNSUPPORTED, "sorted kinds over 2^30 groups or more");
  Scratch& sc = *a.scratch;

  // labels: each row's output row
  auto* inv    = static_cast<uint32_t*>(sc.get((a.table.cap + 1) * sizeof(uint32_t)));
  auto* labels = static_cast<uint32_t*>(sc.get(static_cast<size_t>(n) * sizeof(uint32_t)));
  k_slot_rows<<<grid_of(G, a.num_sms), 256, 0, s>>>(a.map, G, inv);
  GBX_CUDA(cudaGetLastError());
  if (a.plan.key.nwords == 1)
    k_row_labels<1><<<grid_of(n, a.num_sms), 256, 0, s>>>(a.plan, a.table, n, inv, a.max_probes, labels);
  else
    k_row_labels<2><<<grid_of(n, a.num_sms), 256, 0, s>>>(a.plan, a.table, n, inv, a.max_probes, labels);
  GBX_CUDA(cudaGetLastError());
  *launches += 2;

  // records (lo: packed words or split order keys; hi: split labels), their
  // ping-pong copies, tile counts, scan scratch
  const int ntiles    = static_cast<int>((n + kSortTile - 1) / kSortTile);
  const size_t nrec   = static_cast<size_t>(n);
  auto* lo0           = static_cast<uint64_t*>(sc.get(nrec * 8));
  auto* lo1           = static_cast<uint64_t*>(sc.get(nrec * 8));
  uint32_t* hi0       = nullptr;
  uint32_t* hi1       = nullptr;
  const int64_t items = static_cast<int64_t>(ntiles) * 256;
  auto* counts        = static_cast<uint32_t*>(sc.get(static_cast<size_t>(items) * 4));
  auto* offsets       = static_cast<uint32_t*>(sc.get(static_cast<size_t>(items) * 4));
  size_t tb_items = 0, tb_flags = 0;
  GBX_CUDA(scan_exclusive_u32(nullptr, nullptr, items, nullptr, &tb_items, s));
  GBX_CUDA(scan_exclusive_u32(nullptr, nullptr, n + 1, nullptr, &tb_flags, s));
  const size_t tb = std::max(tb_items, tb_flags);
  void* temp      = sc.get(tb);
  auto* bounds    = static_cast<int64_t*>(sc.get(static_cast<size_t>(G) * 3 * sizeof(int64_t)));
  auto* range     = static_cast<Range*>(sc.get(sizeof(Range)));
  uint32_t* flags = nullptr;

  // labels < 2^lbits (G < 2^lbits); packed records use labels 0..G
  const int lbits = std::max(1, bits_for(static_cast<uint64_t>(G)));
  const int pbits = bits_for(static_cast<uint64_t>(G));  // bits of the largest packed label, G
  const int rbits = std::max(1, bits_for(static_cast<uint64_t>(n - 1)));

  GBX_CUDA(cudaFuncSetAttribute(k_sort_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(scatter_smem_bytes(true))));
  GBX_CUDA(cudaFuncSetAttribute(k_sort_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(scatter_smem_bytes(false))));

  // sorts the records on bits [from, to) (split: lo's low lo_bits, then hi's
  // label bits); returns where the result lies and fills `bounds`
  auto sort = [&](bool split, int from, int to, int lo_bits, const Fmt& f) {
    uint64_t *li = lo0, *lout = lo1;
    uint32_t *hin = hi0, *hout = hi1;
    std::vector<int> shifts;
    if (split) {
      for (int b = 0; b < lo_bits; b += 8) shifts.push_back(b);
      for (int b = 0; b < lbits + 2; b += 8) shifts.push_back(64 + b);
    } else {
      for (int b = from; b < to; b += 8) shifts.push_back(b);
    }
    for (int sh : shifts) {
      size_t tbx = tb;
      if (split) {
        k_sort_hist<true><<<ntiles, kSortBlock, 0, s>>>(li, hin, n, sh, ntiles, counts);
        GBX_CUDA(cudaGetLastError());
        GBX_CUDA(scan_exclusive_u32(counts, offsets, items, temp, &tbx, s));
        k_sort_scatter<true><<<ntiles, kSortBlock, scatter_smem_bytes(true), s>>>(li, hin, n, sh, ntiles, offsets,
                                                                                  lout, hout);
      } else {
        k_sort_hist<false><<<ntiles, kSortBlock, 0, s>>>(li, nullptr, n, sh, ntiles, counts);
        GBX_CUDA(cudaGetLastError());
        GBX_CUDA(scan_exclusive_u32(counts, offsets, items, temp, &tbx, s));
        k_sort_scatter<false><<<ntiles, kSortBlock, scatter_smem_bytes(false), s>>>(li, nullptr, n, sh, ntiles,
                                                                                   offsets, lout, nullptr);
      }
      GBX_CUDA(cudaGetLastError());
      *launches += 2 + scan_launches(items);
      std::swap(li, lout);
      std::swap(hin, hout);
    }
    if (split) k_group_bounds<true><<<grid_of(G, a.num_sms), 256, 0, s>>>(li, hin, n, G, f, bounds);
    else k_group_bounds<false><<<grid_of(G, a.num_sms), 256, 0, s>>>(li, nullptr, n, G, f, bounds);
    GBX_CUDA(cudaGetLastError());
    *launches += 1;
    return std::make_pair(li, hin);
  };

  // one sort of a channel's values serves all of its MEDIAN / QUANTILE /
  // NUNIQUE outputs (the caller lists them together)
  int sorted_chan = -1;
  Fmt fmt{};
  int key_bits = 64;
  std::pair<uint64_t*, uint32_t*> sorted{nullptr, nullptr};
  for (const SortedOut& o : a.outs) {
    const Channel& ch = a.plan.chan[o.chan];
    if (o.kind == GBX_AGG_NTH_ELEMENT) {
      // rows, sorted on the label bits alone: row order within a group
      const bool skip = o.null_policy == GBX_NULL_EXCLUDE;
      k_records_packed<<<grid_of(n, a.num_sms), 256, 0, s>>>(ch, n, labels, true, skip, static_cast<uint32_t>(G),
                                                             rbits, 0, lo0, a.status);
      GBX_CUDA(cudaGetLastError());
      *launches += 1;
      sorted_chan = -1;  // the record buffers now hold rows
      Fmt f{false, rbits, 0, (1ULL << rbits) - 1, 0};
      const auto recs = sort(false, rbits, rbits + pbits, 0, f);
      k_nth_element<<<grid_of(G, a.num_sms), 256, 0, s>>>(ch, recs.first, bounds, G, f.vmask, o.nth, o.out_width,
                                                          o.data, o.mask, o.null_count, a.status);
      GBX_CUDA(cudaGetLastError());
      *launches += 1;
      continue;
    }
    if (sorted_chan != o.chan) {
      // the range of the values decides the record format
      GBX_CUDA(cudaMemsetAsync(range, 0, sizeof(Range), s));
      GBX_CUDA(cudaMemsetAsync(&range->kmin, 0xff, sizeof(unsigned long long), s));
      k_value_range<<<grid_of(n, a.num_sms), 256, 0, s>>>(ch, n, labels, range, a.status);
      GBX_CUDA(cudaGetLastError());
      Range h{};
      GBX_CUDA(cudaMemcpyAsync(&h, range, sizeof(Range), cudaMemcpyDeviceToHost, s));
      GBX_CUDA(cudaStreamSynchronize(s));
      const int vbits = h.any ? bits_for(h.kmax - h.kmin) : 0;
      const bool packed = pbits + 1 + vbits <= 64 && !(ch.ptype == P_F32 && h.neg_zero);
      *launches += 2;
      if (packed) {
        k_records_packed<<<grid_of(n, a.num_sms), 256, 0, s>>>(ch, n, labels, false, false,
                                                               static_cast<uint32_t>(G), vbits, h.kmin, lo0,
                                                               a.status);
        fmt      = Fmt{false, vbits + 1, 1ULL << vbits, vbits ? (~0ULL >> (64 - vbits)) : 0, h.kmin};
        key_bits = 64;
        GBX_CUDA(cudaGetLastError());
        sorted = sort(false, 0, pbits + 1 + vbits, 0, fmt);
      } else {
        if (hi0 == nullptr) {
          hi0 = static_cast<uint32_t*>(sc.get(nrec * 4));
          hi1 = static_cast<uint32_t*>(sc.get(nrec * 4));
        }
        k_records_split<<<grid_of(n, a.num_sms), 256, 0, s>>>(ch, n, labels, 1u << (lbits + 1), lo0, hi0,
                                                              a.status);
        GBX_CUDA(cudaGetLastError());
        fmt      = Fmt{true, 0, 0, 0, 0};
        key_bits = 8 * pt_width(ch.ptype);
        sorted   = sort(true, 0, 0, key_bits, fmt);
      }
      sorted_chan = o.chan;
    }
    if (o.kind == GBX_AGG_NUNIQUE) {
      if (flags == nullptr) {
        flags = static_cast<uint32_t*>(sc.get((nrec + 1) * 4));
        GBX_CUDA(cudaMemsetAsync(flags + n, 0, 4, s));  // read by the scan, never counted
      }
      const uint64_t key_mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
      if (fmt.split)
        k_distinct_flags<true><<<grid_of(n, a.num_sms), 256, 0, s>>>(sorted.first, sorted.second, n, key_mask, flags);
      else
        k_distinct_flags<false><<<grid_of(n, a.num_sms), 256, 0, s>>>(sorted.first, nullptr, n, key_mask, flags);
      GBX_CUDA(cudaGetLastError());
      size_t tbx = tb;
      GBX_CUDA(scan_exclusive_u32(flags, flags, n + 1, temp, &tbx, s));
      k_nunique<<<grid_of(G, a.num_sms), 256, 0, s>>>(flags, bounds, G, o.null_policy == GBX_NULL_INCLUDE,
                                                      static_cast<int32_t*>(o.data));
      GBX_CUDA(cudaGetLastError());
      *launches += 2 + scan_launches(n + 1);
    } else {
      const int nq = o.num_quantiles;
      if (nq == 0) continue;
      if (fmt.split)
        k_quantiles<true><<<grid_of(G * nq, a.num_sms), 256, 0, s>>>(
          sorted.first, bounds, G, fmt, ch.ptype, o.quantiles_dev, nq, o.interpolation, static_cast<double*>(o.data),
          o.mask, o.null_count);
      else
        k_quantiles<false><<<grid_of(G * nq, a.num_sms), 256, 0, s>>>(
          sorted.first, bounds, G, fmt, ch.ptype, o.quantiles_dev, nq, o.interpolation, static_cast<double*>(o.data),
          o.mask, o.null_count);
      GBX_CUDA(cudaGetLastError());
      *launches += 1;
    }
  }
}

}  // namespace gbx
