// gbx_scan.cu -- libgbx's own device-wide exclusive scans and the compaction
// of a hash table's occupied slots.
//
// Scans (bucket offsets of the radix passes, partition offsets, per-instance
// group offsets of the batched form) are reduce-then-scan over tiles of
// kScanTile values: one CTA per tile sums its tile, one CTA scans the tile
// sums, and one CTA per tile scans its tile with that base.  The inputs are
// at most a few tens of MB (6.2M u32 for the 100M-row radix passes), so the
// extra read of the tiles costs microseconds; a single tile (the common
// small case) is one launch.
//
// Compaction lists the occupied slots of a table (the reference's
// retrieve_all of cuco::static_set, cpp/src/groupby/hash/groupby.cu:510-520):
// each warp ballots 32 slots, a block scan of the warp counts places them,
// and one atomic per block and sweep reserves the block's output positions.
// The output order of the groups is therefore unspecified (as it is in the
// reference).
#include <cuda_runtime.h>

#include <algorithm>

#include "gbx_kernels.hpp"
#include "gbx_scan.hpp"

namespace gbx {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile  = kScanBlock * kScanItems;

// Exclusive scan of one value per thread across the block; returns the
// block total through *total.  `warp_sums` holds kScanBlock / 32 values.
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* warp_sums, T* total)
{
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  T inc          = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const T o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    constexpr int kWarps = kScanBlock / 32;
    T w                  = lane < kWarps ? warp_sums[lane] : T(0);
    T wi                 = w;
#pragma unroll
    for (int d = 1; d < kWarps; d <<= 1) {
      const T o = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += o;
    }
    if (lane < kWarps) warp_sums[lane] = wi - w;  // exclusive warp offsets
    if (lane == kWarps - 1) *total = wi;
  }
  __syncthreads();
  const T r = warp_sums[warp] + inc - v;
  __syncthreads();  // warp_sums may be reused by the caller
  return r;
}

// Loads tile `b` of `in` (n values) into registers in blocked order (thread t
// holds values t*kScanItems ..), through shared memory so that the global
// loads are coalesced.  Values past n read as 0.
template <class T>
__device__ __forceinline__ void load_tile(const T* in, int64_t n, int64_t b, T (&x)[kScanItems], T* stage)
{
  const int64_t base = b * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j       = i * kScanBlock + threadIdx.x;
    const int64_t idx = base + j;
    stage[j + j / 32] = idx < n ? in[idx] : T(0);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j = threadIdx.x * kScanItems + i;
    x[i]        = stage[j + j / 32];
  }
  __syncthreads();
}

template <class T>
__device__ __forceinline__ void store_tile(T* out, int64_t n, int64_t b, const T (&x)[kScanItems], T* stage)
{
  const int64_t base = b * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j       = threadIdx.x * kScanItems + i;
    stage[j + j / 32] = x[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j       = i * kScanBlock + threadIdx.x;
    const int64_t idx = base + j;
    if (idx < n) out[idx] = stage[j + j / 32];
  }
}

template <class T>
struct ScanSmem {
  T stage[kScanTile + kScanTile / 32];
  T warp_sums[kScanBlock / 32];
  T total;
};

// Tile sums.
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_reduce(const T* __restrict__ in, int64_t n, T* __restrict__ sums)
{
  __shared__ ScanSmem<T> sm;
  T x[kScanItems];
  load_tile(in, n, blockIdx.x, x, sm.stage);
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) s += x[i];
  block_exclusive_scan<T>(s, sm.warp_sums, &sm.total);
  if (threadIdx.x == 0) sums[blockIdx.x] = sm.total;
}

// Exclusive scan of `n` values in place by one CTA, tile after tile with a
// running carry; the grand total goes to sums[n].
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_single(T* __restrict__ sums, int64_t n)
{
  __shared__ ScanSmem<T> sm;
  T carry = 0;
  for (int64_t b = 0; b * kScanTile < n; ++b) {
    T x[kScanItems];
    load_tile(sums, n, b, x, sm.stage);
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) s += x[i];
    T run = block_exclusive_scan<T>(s, sm.warp_sums, &sm.total) + carry;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const T v = x[i];
      x[i]      = run;
      run += v;
    }
    store_tile(sums, n, b, x, sm.stage);
    carry += sm.total;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[n] = carry;
}

// Tile b's exclusive scan plus its base sums[b].
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_down(const T* __restrict__ in, T* __restrict__ out, int64_t n,
                                                        const T* __restrict__ sums)
{
  __shared__ ScanSmem<T> sm;
  T x[kScanItems];
  load_tile(in, n, blockIdx.x, x, sm.stage);
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) s += x[i];
  T run = block_exclusive_scan<T>(s, sm.warp_sums, &sm.total) + sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const T v = x[i];
    x[i]      = run;
    run += v;
  }
  store_tile(out, n, blockIdx.x, x, sm.stage);
}

// One tile: the whole scan in one CTA (out may alias in).
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_one_tile(const T* __restrict__ in, T* __restrict__ out, int64_t n)
{
  __shared__ ScanSmem<T> sm;
  T x[kScanItems];
  load_tile(in, n, 0, x, sm.stage);
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) s += x[i];
  T run = block_exclusive_scan<T>(s, sm.warp_sums, &sm.total);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const T v = x[i];
    x[i]      = run;
    run += v;
  }
  store_tile(out, n, 0, x, sm.stage);
}

template <class T>
cudaError_t scan_impl(const T* in, T* out, int64_t n, void* temp, size_t* temp_bytes, cudaStream_t st)
{
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  const size_t need   = static_cast<size_t>(std::max<int64_t>(tiles, 1) + 1) * sizeof(T);
  if (temp == nullptr) {
    *temp_bytes = need;
    return cudaSuccess;
  }
  if (*temp_bytes < need) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  if (tiles == 1) {
    k_scan_one_tile<T><<<1, kScanBlock, 0, st>>>(in, out, n);
    return cudaGetLastError();
  }
  T* sums = static_cast<T*>(temp);
  k_scan_reduce<T><<<static_cast<unsigned>(tiles), kScanBlock, 0, st>>>(in, n, sums);
  k_scan_single<T><<<1, kScanBlock, 0, st>>>(sums, tiles);
  k_scan_down<T><<<static_cast<unsigned>(tiles), kScanBlock, 0, st>>>(in, out, n, sums);
  return cudaGetLastError();
}

// ----------------------------------------------------------- compaction

constexpr int kCompactBlock = 256;

template <int NW>
__global__ void __launch_bounds__(kCompactBlock) k_compact_occupied(const uint64_t* __restrict__ keys,
                                                                 const uint32_t* __restrict__ special_used,
                                                                 uint64_t cap, uint32_t* __restrict__ map,
                                                                 unsigned long long* __restrict__ count)
{
  __shared__ uint32_t warp_cnt[kCompactBlock / 32];
  __shared__ unsigned long long block_base;
  const int lane   = threadIdx.x & 31;
  const int warp   = threadIdx.x >> 5;
  const uint64_t n = cap + 1;
  for (uint64_t s0 = static_cast<uint64_t>(blockIdx.x) * kCompactBlock; s0 < n;
       s0 += static_cast<uint64_t>(gridDim.x) * kCompactBlock) {
    const uint64_t s = s0 + threadIdx.x;
    bool occ         = false;
    if (s < cap) {
      if constexpr (NW == 1) {
        occ = __ldg(keys + s) != kEmptyWord;
      } else {
        const ulonglong2 k = __ldg(reinterpret_cast<const ulonglong2*>(keys) + s);
        occ                = !(k.x == kEmptyWord && k.y == kEmptyWord);
      }
    } else if (s == cap) {
      occ = *special_used != 0;
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) warp_cnt[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
#pragma unroll
      for (int w = 0; w < kCompactBlock / 32; ++w) {
        const uint32_t c = warp_cnt[w];
        warp_cnt[w]      = tot;
        tot += c;
      }
      block_base = tot ? atomicAdd(count, static_cast<unsigned long long>(tot)) : 0ull;
    }
    __syncthreads();
    if (occ) map[block_base + warp_cnt[warp] + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint32_t>(s);
    __syncthreads();
  }
}

}  // namespace

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, void* temp, size_t* temp_bytes,
                               cudaStream_t st)
{
  return scan_impl<uint32_t>(in, out, n, temp, temp_bytes, st);
}

cudaError_t scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, void* temp, size_t* temp_bytes,
                               cudaStream_t st)
{
  return scan_impl<long long>(reinterpret_cast<const long long*>(in), reinterpret_cast<long long*>(out), n, temp,
                              temp_bytes, st);
}

int scan_launches(int64_t n) { return n <= 0 ? 0 : n <= kScanTile ? 1 : 3; }

cudaError_t compact_occupied(const TableRef& t, int nwords, uint32_t* map, int64_t* num_selected, int num_sms,
                             cudaStream_t st)
{
  cudaError_t e = cudaMemsetAsync(num_selected, 0, sizeof(int64_t), st);
  if (e != cudaSuccess) return e;
  const uint64_t n    = t.cap + 1;
  const uint64_t want = (n + kCompactBlock - 1) / kCompactBlock;
  const int grid      = static_cast<int>(std::min<uint64_t>(want, static_cast<uint64_t>(num_sms) * 8));
  auto* cnt           = reinterpret_cast<unsigned long long*>(num_selected);
  if (nwords == 1) k_compact_occupied<1><<<grid, kCompactBlock, 0, st>>>(t.keys, t.special_used, t.cap, map, cnt);
  else k_compact_occupied<2><<<grid, kCompactBlock, 0, st>>>(t.keys, t.special_used, t.cap, map, cnt);
  return cudaGetLastError();
}

const void* compact_kernel(int nwords)
{
  return nwords == 1 ? reinterpret_cast<const void*>(k_compact_occupied<1>)
                     : reinterpret_cast<const void*>(k_compact_occupied<2>);
}

}  // namespace gbx
