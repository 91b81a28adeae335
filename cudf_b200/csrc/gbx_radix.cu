// gbx_radix.cu -- coalesced radix partitioning of the rows into hash buckets
// (the partitioned path's scatter for many buckets).
//
// A one-pass scatter into 2^bits buckets sends each warp's 32 rows to 32
// far-apart places once bits is large, so every 32-byte sector it writes is
// partial and is filled from DRAM before the write lands (3.3x the
// algorithmic traffic measured with ncu at 2^18 buckets), and every row waits
// for a global cursor atomic.  Here the bucket id is instead split into
// digits of at most 8 bits and the rows are moved once per digit, least
// significant digit first, by a stable counting sort: per 4,096-row tile a
// histogram of the digit, one exclusive scan over (digit, tile), and a
// scatter in which each row's position is its tile's offset for the digit
// plus its rank among the tile's rows of that digit.  A tile's rows of one
// digit land next to each other, so sectors are written whole while they sit
// in L2, and no global atomics are used.  After the last pass the rows are in
// bucket order, stable within a bucket, exactly where the bucket offsets of
// the histogram (k_part_hist) place them.

#include <algorithm>

#include "gbx_scan.hpp"
#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kRadixBlock  = 256;
constexpr int kRadixWarps  = kRadixBlock / 32;
constexpr int kRowsPerWarp = 512;  // 16 batches of 32
constexpr int kTileRows    = kRadixWarps * kRowsPerWarp;
constexpr int kMaxRadix    = 256;
constexpr int kLoadGroup   = 8;  // 32-row batches whose loads a warp has in flight together

struct Digit {
  int bits;   // bucket id = top `bits` bits of the key hash
  int shift;  // this pass's digit = (bucket >> shift) & (radix - 1)
  int width;  // digit bits (<= 8)
};

template <int NW>
__device__ __forceinline__ uint32_t digit_of(const uint64_t (&k)[NW], const Digit& dg)
{
  const uint64_t h = hash_key<NW>(k);
  const uint32_t b = dg.bits == 0 ? 0u : static_cast<uint32_t>(h >> (64 - dg.bits));
  return (b >> dg.shift) & ((1u << dg.width) - 1u);
}

// Row r of the pass's source: the caller's columns (first pass: rows with a
// null key under EXCLUDE are dropped, values resolved) or the previous pass's
// bucket copies.
template <int NW, bool FROM_COLUMNS>
struct PassSource {
  const Plan* plan;
  const PartBufs* in;
  __device__ __forceinline__ bool key(int64_t r, uint64_t (&k)[NW]) const
  {
    if constexpr (FROM_COLUMNS) {
      return pack_key<NW>(plan->key, r, k);
    } else {
#pragma unroll
      for (int w = 0; w < NW; ++w) k[w] = __ldg(in->keys[w] + r);
      return true;
    }
  }
  __device__ __forceinline__ bool value(int c, int64_t r, uint64_t& b, int32_t* status) const
  {
    if constexpr (FROM_COLUMNS) {
      return RowSource{plan}.value(c, r, b, status);
    } else {
      const PartCol& pc = in->col[c];
      b                 = load_bits(pc.vals, r, pc.width);
      return pc.valid == nullptr || __ldg(pc.valid + r) != 0;
    }
  }
};

__device__ __forceinline__ int64_t source_rows(int64_t n, const uint32_t* n_active, bool from_columns)
{
  return from_columns ? n : static_cast<int64_t>(*n_active);
}

// counts[d * ntiles + t] = rows of tile t whose digit is d; when
// bucket_counts is set, also adds every row to its bucket's count there
// (the bucket histogram of the partitioned path, warp-aggregated).  PLAIN (a
// first pass over a single plain 8-byte key column without nulls): the key
// words are read straight from in.keys[0], the caller's column, n rows.
template <int NW, bool FROM_COLUMNS, bool PLAIN = false>
__global__ void __launch_bounds__(kRadixBlock) k_radix_hist(const __grid_constant__ Plan plan,
                                                            const __grid_constant__ PartBufs in, int64_t n,
                                                            const uint32_t* n_active, const Digit dg, int ntiles,
                                                            uint32_t* counts, uint32_t* bucket_counts)
{
  __shared__ uint32_t hist[kMaxRadix];
  const int radix = 1 << dg.width;
  for (int i = threadIdx.x; i < radix; i += kRadixBlock) hist[i] = 0;
  __syncthreads();
  const PassSource<NW, FROM_COLUMNS && !PLAIN> src{&plan, &in};
  const int64_t rows = source_rows(n, n_active, FROM_COLUMNS);
  const int lane     = threadIdx.x & 31;
  const int warp     = threadIdx.x >> 5;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTileRows + warp * kRowsPerWarp;
  for (int j0 = 0; j0 < kRowsPerWarp / 32; j0 += kLoadGroup) {
    // the group's loads are issued before any of them is used
    uint64_t k[kLoadGroup][NW];
    bool act[kLoadGroup];
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const int64_t r = base + (j0 + u) * 32 + lane;
      act[u]          = r < rows && src.key(r, k[u]);
    }
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const uint64_t h   = act[u] ? hash_key<NW>(k[u]) : 0;
      const uint32_t bkt = dg.bits == 0 ? 0u : static_cast<uint32_t>(h >> (64 - dg.bits));
      const uint32_t d   = (bkt >> dg.shift) & ((1u << dg.width) - 1u);
      if (act[u]) atomicAdd(&hist[d], 1u);  // shared 32-bit atomics: cheaper than grouping the warp first
      if (bucket_counts != nullptr) {
        const uint32_t pb = __match_any_sync(kFull, act[u] ? bkt : 0xffffffffu);
        if (act[u] && lane == __ffs(pb) - 1) atomicAdd(bucket_counts + bkt, static_cast<uint32_t>(__popc(pb)));
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < radix; i += kRadixBlock)
    counts[static_cast<size_t>(i) * ntiles + blockIdx.x] = hist[i];
}

// Shared memory of k_radix_scatter (dynamic: more than the 48 KB static limit).
struct ScatterSmem {
  uint64_t stage[kTileRows];              // one column of the tile, in digit order
  uint32_t cnt[kRadixWarps][kMaxRadix];   // per warp: rows of each digit, then its first local position
  uint32_t tstart[kMaxRadix];             // first local position of each digit in the tile
  uint32_t goff[kMaxRadix];               // first global position of the tile's rows of each digit
  uint16_t lpos[kTileRows];               // local position of tile row (warp, batch, lane); 0xffff: dropped
  uint32_t gp[kTileRows];                 // output row of each local position
  uint8_t vstage[kTileRows];              // validity of the staged values
  uint32_t active;                        // rows of the tile kept
};
constexpr size_t kScatterSmem = sizeof(ScatterSmem);

// The first pass: moves the rows of tile blockIdx.x of the caller's columns
// to offsets[d * ntiles + t] + their rank among the tile's rows of digit d
// (tile order: warp, then batch, then lane).  Rows are first ranked in digit
// order inside the tile (local positions); each column is then staged in
// shared memory at those positions and written out by consecutive threads,
// so a digit's run of rows is stored by consecutive lanes into consecutive
// addresses.
template <int NW, bool FROM_COLUMNS = true>
__global__ void __launch_bounds__(kRadixBlock, 3) k_radix_scatter(const __grid_constant__ Plan plan,
                                                               const __grid_constant__ PartBufs in, int64_t n,
                                                               const uint32_t* n_active, const Digit dg, int ntiles,
                                                               const uint32_t* __restrict__ offsets,
                                                               const __grid_constant__ PartBufs out, int32_t* status)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem& sm = *reinterpret_cast<ScatterSmem*>(smem_raw);
  const int radix = 1 << dg.width;
  for (int i = threadIdx.x; i < kRadixWarps * kMaxRadix; i += kRadixBlock) (&sm.cnt[0][0])[i] = 0;
  // the tile's first output row of each digit, loaded now so that the load
  // overlaps the ranking (one digit per thread)
  static_assert(kRadixBlock >= kMaxRadix, "one digit per thread");
  const uint32_t my_goff =
    threadIdx.x < radix ? __ldg(offsets + static_cast<size_t>(threadIdx.x) * ntiles + blockIdx.x) : 0u;
  __syncthreads();
  const PassSource<NW, FROM_COLUMNS> src{&plan, &in};
  const int64_t rows = source_rows(n, n_active, FROM_COLUMNS);
  const int lane     = threadIdx.x & 31;
  const int warp     = threadIdx.x >> 5;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTileRows + warp * kRowsPerWarp;
  const uint32_t lt  = (1u << lane) - 1u;

  // rows of each digit per warp (each warp owns its row of cnt); each row's
  // digit is kept in lpos (0xffff: row dropped) until its position is known
  for (int j0 = 0; j0 < kRowsPerWarp / 32; j0 += kLoadGroup) {
    uint64_t k[kLoadGroup][NW];
    bool act[kLoadGroup];
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const int64_t r = base + (j0 + u) * 32 + lane;
      act[u]          = r < rows && src.key(r, k[u]);
    }
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const int row       = warp * kRowsPerWarp + (j0 + u) * 32 + lane;
      const uint32_t d    = act[u] ? digit_of<NW>(k[u], dg) : 0u;
      const uint32_t pe   = digit_peers(d, dg.width, __ballot_sync(kFull, act[u]));
      const uint32_t prev = act[u] ? sm.cnt[warp][d] : 0u;
      // the row's rank among its warp's rows of its digit, and the digit
      // (in vstage, unused until the columns are staged)
      sm.lpos[row]   = static_cast<uint16_t>(act[u] ? prev + static_cast<uint32_t>(__popc(pe & lt)) : 0xffffu);
      sm.vstage[row] = static_cast<uint8_t>(d);
      __syncwarp();
      if (act[u] && (pe & lt) == 0) sm.cnt[warp][d] = prev + static_cast<uint32_t>(__popc(pe));
      __syncwarp();
    }
  }
  __syncthreads();
  // digit totals of the tile -> first local position of each digit (warp 0
  // scans 8 digits per lane); global offsets of the tile's runs
  if (warp == 0) {
    uint32_t tot[kMaxRadix / 32];
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < kMaxRadix / 32; ++q) {
      const int d = lane * (kMaxRadix / 32) + q;
      uint32_t c  = 0;
      if (d < radix)
        for (int w = 0; w < kRadixWarps; ++w) c += sm.cnt[w][d];
      tot[q] = c;
      sum += c;
    }
    uint32_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += v;
    }
    uint32_t run = incl - sum;
#pragma unroll
    for (int q = 0; q < kMaxRadix / 32; ++q) {
      const int d = lane * (kMaxRadix / 32) + q;
      if (d < radix) sm.tstart[d] = run;
      run += tot[q];
    }
    if (lane == 31) sm.active = incl;
  }
  __syncthreads();
  if (threadIdx.x < radix) {
    const int d  = threadIdx.x;
    sm.goff[d]   = my_goff;
    uint32_t run = sm.tstart[d];
    for (int w = 0; w < kRadixWarps; ++w) {
      const uint32_t c = sm.cnt[w][d];
      sm.cnt[w][d]     = run;
      run += c;
    }
  }
  __syncthreads();
  // local positions (the rank comes back from lpos, which then takes the
  // position, the digit from vstage) and the output row of each; key word 0
  // staged on the way
  for (int j0 = 0; j0 < kRowsPerWarp / 32; j0 += kLoadGroup) {
    uint64_t k0[kLoadGroup];
    uint32_t rr[kLoadGroup];
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const int row = warp * kRowsPerWarp + (j0 + u) * 32 + lane;
      rr[u]         = sm.lpos[row];
      k0[u]         = 0;
      if (rr[u] != 0xffffu) {
        uint64_t k[NW];
        src.key(base + (j0 + u) * 32 + lane, k);
        k0[u] = k[0];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadGroup; ++u) {
      const int row = warp * kRowsPerWarp + (j0 + u) * 32 + lane;
      if (rr[u] != 0xffffu) {
        const uint32_t d  = sm.vstage[row];
        const uint32_t lp = sm.cnt[warp][d] + rr[u];
        sm.lpos[row]      = static_cast<uint16_t>(lp);
        sm.gp[lp]         = sm.goff[d] + (lp - sm.tstart[d]);
        sm.stage[lp]      = k0[u];
      }
    }
  }
  __syncthreads();
  const uint32_t active = sm.active;
  auto global_pos = [&](uint32_t i) -> uint32_t { return sm.gp[i]; };
  for (uint32_t i = threadIdx.x; i < active; i += kRadixBlock)
    const_cast<uint64_t*>(out.keys[0])[global_pos(i)] = sm.stage[i];
  __syncthreads();
  // remaining key word, then every channel's values and validity
  for (int col = 1; col < NW + plan.nchan; ++col) {
    const int c = col - NW;
    for (int j0 = 0; j0 < kRowsPerWarp / 32; j0 += kLoadGroup) {
      uint32_t lp[kLoadGroup];
      uint64_t val[kLoadGroup];
      bool v[kLoadGroup];
#pragma unroll
      for (int u = 0; u < kLoadGroup; ++u) {
        lp[u]  = sm.lpos[warp * kRowsPerWarp + (j0 + u) * 32 + lane];
        val[u] = 0;
        v[u]   = false;
        if (lp[u] == 0xffffu) continue;
        const int64_t r = base + (j0 + u) * 32 + lane;
        if (col < NW) {
          uint64_t k[NW];
          src.key(r, k);
          val[u] = k[col & (NW - 1)];
          v[u]   = true;
        } else {
          v[u] = src.value(c, r, val[u], status);
        }
      }
#pragma unroll
      for (int u = 0; u < kLoadGroup; ++u) {
        if (lp[u] == 0xffffu) continue;
        sm.stage[lp[u]]  = v[u] ? val[u] : 0;
        sm.vstage[lp[u]] = v[u] ? 1 : 0;
      }
    }
    __syncthreads();
    if (col < NW) {
      for (uint32_t i = threadIdx.x; i < active; i += kRadixBlock)
        const_cast<uint64_t*>(out.keys[col & (NW - 1)])[global_pos(i)] = sm.stage[i];
    } else {
      const PartCol& pc = out.col[c];
      for (uint32_t i = threadIdx.x; i < active; i += kRadixBlock) {
        const uint32_t at = global_pos(i);
        store_bits(const_cast<void*>(pc.vals), at, pc.width, sm.stage[i]);
        if (pc.valid != nullptr) const_cast<uint8_t*>(pc.valid)[at] = sm.vstage[i];
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- bulk passes
//
// Passes after the first read the previous pass's copies, where each column
// of a tile is one contiguous run of bytes.  k_radix_scatter_bulk moves such
// a column into shared memory with one cp.async.bulk (the copy engine, not
// the threads, performs the loads; completion is counted on an mbarrier),
// two columns in flight at a time: while a column is written out the next
// but one is already arriving.  The digits come from the key words in shared
// memory, every local position's output row is computed once, and each
// column's write-out is then a shared-memory gather by local position and a
// store to consecutive rows of a digit's run.  A tile that is not full, or a
// column that is not 16-byte aligned, is copied by the threads instead.

struct BulkSmem {
  unsigned long long raw[2][kTileRows];  // two column buffers, in tile-row order
  uint32_t gp[kTileRows];                // output row of local position i
  uint16_t src[kTileRows];               // tile row at local position i
  uint8_t dig[kTileRows];                // digit of tile row r
  uint16_t rk[kTileRows];                // rank of tile row r among its warp's rows of its digit
  uint32_t cnt[kRadixWarps][kMaxRadix];  // per warp: rows of each digit, then its first local position
  uint32_t tstart[kMaxRadix];            // first local position of each digit in the tile
  uint32_t goff[kMaxRadix];              // first output row of the tile's rows of each digit
  unsigned long long bar[2];             // completion of each buffer's copy
};
constexpr size_t kBulkSmem = sizeof(BulkSmem);

// ~1 s at the B200's clocks: a wait for a copy this long means the copy is
// not coming; the kernel then reports S_SPIN_LIMIT instead of hanging.
constexpr long long kCopyWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok)
    : "r"(bar), "r"(parity)
    : "memory");
  return ok != 0;
}
// Waits for phase `parity` of a barrier to complete, for at most
// kCopyWaitCycles; false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kCopyWaitCycles) return false;
  return true;
}

// dst[at[k]] = column[from[k]] for this thread's local positions (elements
// of type T; from[k] == all-ones: none), all gathers issued before the stores.
template <class T, int KPER>
__device__ __forceinline__ void gather_column(const unsigned long long* column, const uint32_t (&from)[KPER],
                                              const uint32_t (&at)[KPER], unsigned char* dst)
{
  const T* s = reinterpret_cast<const T*>(column);
  T* d       = reinterpret_cast<T*>(dst);
  T v[KPER];
#pragma unroll
  for (int k = 0; k < KPER; ++k) v[k] = from[k] != 0xffffffffu ? s[from[k]] : T(0);
#pragma unroll
  for (int k = 0; k < KPER; ++k)
    if (from[k] != 0xffffffffu) d[at[k]] = v[k];
}

// Column j of a pass: key words first, then each channel's values followed
// by its validity bytes when it has them.
struct PassCol {
  const unsigned char* src;
  unsigned char* dst;
  int width;
  int chan;       // channel of a value or validity column, else -1
  bool validity;  // the channel's validity bytes
};
// The columns follow `out`: a channel has a validity column when its copies
// keep validity bytes.
template <int NW>
__device__ __forceinline__ PassCol pass_col(const Plan& plan, const PartBufs& in, const PartBufs& out, int j)
{
  if (j < NW)
    return PassCol{reinterpret_cast<const unsigned char*>(in.keys[j]),
                   const_cast<unsigned char*>(reinterpret_cast<const unsigned char*>(out.keys[j])), 8, -1, false};
  j -= NW;
  for (int c = 0; c < plan.nchan; ++c) {
    const PartCol& a = in.col[c];
    const PartCol& b = out.col[c];
    if (j == 0)
      return PassCol{static_cast<const unsigned char*>(a.vals),
                     static_cast<unsigned char*>(const_cast<void*>(b.vals)), b.width, c, false};
    --j;
    if (b.valid != nullptr) {
      if (j == 0) return PassCol{a.valid, const_cast<uint8_t*>(b.valid), 1, c, true};
      --j;
    }
  }
  return PassCol{nullptr, nullptr, 0, -1, false};
}

// `first_pass`: `in` points at the caller's columns themselves (a plain
// 8-byte key column without nulls, value columns without dictionaries, each
// pointer already advanced by its column's offset), all n rows are kept and
// the validity bytes come from the channels' bitmasks; otherwise `in` holds
// the previous pass's copies and *n_active rows.
template <int NW>
__global__ void __launch_bounds__(kRadixBlock, 2) k_radix_scatter_bulk(const __grid_constant__ Plan plan,
                                                                    const __grid_constant__ PartBufs in,
                                                                    const uint32_t* n_active, int64_t n,
                                                                    bool first_pass, const Digit dg,
                                                                    const uint32_t* __restrict__ offsets,
                                                                    int ntiles,
                                                                    const __grid_constant__ PartBufs out,
                                                                    int32_t* status)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BulkSmem& sm        = *reinterpret_cast<BulkSmem*>(smem_raw);
  const int64_t rows  = first_pass ? n : static_cast<int64_t>(*n_active);
  const int64_t start = static_cast<int64_t>(blockIdx.x) * kTileRows;
  if (start >= rows) return;  // an empty tile: nothing to move
  const int nrows = static_cast<int>(rows - start < kTileRows ? rows - start : kTileRows);
  const int radix = 1 << dg.width;
  const int lane  = threadIdx.x & 31;
  const int warp  = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t bar[2] = {smem_addr(&sm.bar[0]), smem_addr(&sm.bar[1])};

  int ncol  = NW;
  bool bulk = nrows == kTileRows;
  for (int c = 0; c < plan.nchan; ++c) ncol += out.col[c].valid != nullptr ? 2 : 1;
  for (int j = 0; j < ncol; ++j) {
    const PassCol pc = pass_col<NW>(plan, in, out, j);
    if (first_pass && pc.validity) continue;  // filled from the bitmask
    bulk = bulk && (reinterpret_cast<uintptr_t>(pc.src) & 15u) == 0;
  }

  if (threadIdx.x == 0 && bulk) {
    mbar_init(bar[0]);
    mbar_init(bar[1]);
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < kRadixWarps * kMaxRadix; i += kRadixBlock) (&sm.cnt[0][0])[i] = 0;
  // the tile's first output row of each digit, loaded now so that the load
  // overlaps the copies and the ranking (one digit per thread)
  static_assert(kRadixBlock >= kMaxRadix, "one digit per thread");
  const uint32_t my_goff =
    threadIdx.x < radix ? __ldg(offsets + static_cast<size_t>(threadIdx.x) * ntiles + blockIdx.x) : 0u;
  __syncthreads();

  uint32_t parity  = 0;  // bit b: phase of buffer b's next completion
  uint32_t pending = 0;  // bit b: a bulk copy into buffer b not yet waited for
  // column j into buffer b (all threads call it right after a barrier that
  // freed the buffer)
  auto issue = [&](int j, int b) {
    const PassCol pc = pass_col<NW>(plan, in, out, j);
    if (first_pass && pc.validity) {
      // validity bytes of the caller's column from its bitmask
      const Channel& ch = plan.chan[pc.chan];
      unsigned char* d  = reinterpret_cast<unsigned char*>(sm.raw[b]);
      for (int i = threadIdx.x; i < nrows; i += kRadixBlock) d[i] = bit_valid(ch.mask, start + i + ch.offset) ? 1 : 0;
    } else if (bulk) {
      if (threadIdx.x == 0) {
        const uint32_t bytes = static_cast<uint32_t>(kTileRows) * pc.width;
        fence_proxy_async();  // the threads' reads of the buffer come first
        mbar_expect_tx(bar[b], bytes);
        bulk_copy_g2s(smem_addr(sm.raw[b]), pc.src + start * pc.width, bytes, bar[b]);
      }
      pending |= 1u << b;
    } else {
      unsigned char* d = reinterpret_cast<unsigned char*>(sm.raw[b]);
      for (int i = threadIdx.x; i < nrows; i += kRadixBlock) {
        const int64_t r = start + i;
        switch (pc.width) {
          case 1: d[i] = __ldg(pc.src + r); break;
          case 2: reinterpret_cast<uint16_t*>(d)[i] = __ldg(reinterpret_cast<const uint16_t*>(pc.src) + r); break;
          case 4: reinterpret_cast<uint32_t*>(d)[i] = __ldg(reinterpret_cast<const uint32_t*>(pc.src) + r); break;
          default:
            reinterpret_cast<unsigned long long*>(d)[i] =
              __ldg(reinterpret_cast<const unsigned long long*>(pc.src) + r);
            break;
        }
      }
    }
  };
  // buffer b's column is in shared memory (uniform result: false when a copy
  // did not arrive in time)
  auto wait = [&](int b) -> bool {
    bool got = true;
    if (pending & (1u << b)) {  // a bulk copy (thread-filled buffers only need the barrier)
      got = mbar_wait_bounded(bar[b], (parity >> b) & 1u);
      if (got) {
        parity ^= 1u << b;
        pending &= ~(1u << b);
      }
    }
    return __syncthreads_and(got) != 0;
  };
  auto give_up = [&]() {
    if (threadIdx.x == 0) atomicOr(status, S_SPIN_LIMIT);
    for (int b = 0; b < 2; ++b)
      if (pending & (1u << b)) (void)mbar_wait_bounded(bar[b], (parity >> b) & 1u);
  };

  issue(0, 0);
  if (ncol > 1) issue(1, 1);
  bool ok = wait(0);
  if (ok && NW == 2) ok = wait(1);
  if (!ok) {
    give_up();
    return;
  }

  // per warp: rows of each digit; each row's digit and its rank among the
  // warp's rows of that digit kept (stable: batch, then lane order)
  for (int j0 = 0; j0 < kRowsPerWarp / 32; ++j0) {
    const int r    = warp * kRowsPerWarp + j0 * 32 + lane;
    const bool act = r < nrows;
    uint64_t k[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = act ? sm.raw[w][r] : 0;
    const uint32_t d    = act ? digit_of<NW>(k, dg) : 0u;
    const uint32_t pe   = digit_peers(d, dg.width, __ballot_sync(kFull, act));
    const uint32_t prev = act ? sm.cnt[warp][d] : 0u;
    if (act) {
      sm.dig[r] = static_cast<uint8_t>(d);
      sm.rk[r]  = static_cast<uint16_t>(prev + static_cast<uint32_t>(__popc(pe & lt)));
    }
    __syncwarp();
    if (act && (pe & lt) == 0) sm.cnt[warp][d] = prev + static_cast<uint32_t>(__popc(pe));
    __syncwarp();
  }
  __syncthreads();
  // digit totals -> first local position of each digit (warp 0, 8 digits a lane)
  if (warp == 0) {
    uint32_t tot[kMaxRadix / 32];
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < kMaxRadix / 32; ++q) {
      const int d = lane * (kMaxRadix / 32) + q;
      uint32_t c  = 0;
      if (d < radix)
        for (int w = 0; w < kRadixWarps; ++w) c += sm.cnt[w][d];
      tot[q] = c;
      sum += c;
    }
    uint32_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += v;
    }
    uint32_t run = incl - sum;
#pragma unroll
    for (int q = 0; q < kMaxRadix / 32; ++q) {
      const int d = lane * (kMaxRadix / 32) + q;
      if (d < radix) sm.tstart[d] = run;
      run += tot[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < radix) {
    const int d  = threadIdx.x;
    sm.goff[d]   = my_goff;
    uint32_t run = sm.tstart[d];
    for (int w = 0; w < kRadixWarps; ++w) {
      const uint32_t c = sm.cnt[w][d];
      sm.cnt[w][d]     = run;
      run += c;
    }
  }
  __syncthreads();
  // local position of every row (stable: warp, batch, lane order), with the
  // tile row and the output row stored at it
  for (int j0 = 0; j0 < kRowsPerWarp / 32; ++j0) {
    const int r = warp * kRowsPerWarp + j0 * 32 + lane;
    if (r < nrows) {
      const uint32_t d  = sm.dig[r];
      const uint32_t lp = sm.cnt[warp][d] + sm.rk[r];
      sm.src[lp]        = static_cast<uint16_t>(r);
      sm.gp[lp]         = sm.goff[d] + (lp - sm.tstart[d]);
    }
  }
  __syncthreads();

  // this thread's local positions i = threadIdx.x + k * kRadixBlock: tile row
  // and output row, kept in registers for every column (kNoRow: past the tile)
  constexpr int kPer = kTileRows / kRadixBlock;
  constexpr uint32_t kNoRow = 0xffffffffu;
  uint32_t from[kPer], at[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int i = threadIdx.x + k * kRadixBlock;
    from[k]     = i < nrows ? sm.src[i] : kNoRow;
    at[k]       = i < nrows ? sm.gp[i] : 0u;
  }

  for (int j = 0; j < ncol; ++j) {
    const int b = j & 1;
    if (j >= NW) {  // the key words were waited for before the ranking
      if (!wait(b)) {
        give_up();
        return;
      }
    }
    const PassCol pc = pass_col<NW>(plan, in, out, j);
    switch (pc.width) {
      case 1: gather_column<uint8_t, kPer>(sm.raw[b], from, at, pc.dst); break;
      case 2: gather_column<uint16_t, kPer>(sm.raw[b], from, at, pc.dst); break;
      case 4: gather_column<uint32_t, kPer>(sm.raw[b], from, at, pc.dst); break;
      default: gather_column<unsigned long long, kPer>(sm.raw[b], from, at, pc.dst); break;
    }
    __syncthreads();  // buffer b is free again
    if (j + 2 < ncol) issue(j + 2, b);
  }
}

}  // namespace

size_t part_radix_count_bytes(int64_t n)
{
  const int64_t ntiles = (n + kTileRows - 1) / kTileRows;
  return static_cast<size_t>(std::max<int64_t>(ntiles, 1)) * kMaxRadix * sizeof(uint32_t);
}

cudaError_t part_radix_temp_bytes(int64_t n, size_t* temp_bytes)
{
  const int64_t ntiles = (n + kTileRows - 1) / kTileRows;
  const int items      = static_cast<int>(std::max<int64_t>(ntiles, 1) * kMaxRadix);
  return scan_exclusive_u32(nullptr, nullptr, items, nullptr, temp_bytes, cudaStream_t(nullptr));
}

namespace {
// Digit of pass i (least significant first) of a `bits`-bit bucket id.
Digit pass_digit(int bits, int i)
{
  const int passes = (bits + 7) / 8;
  Digit dg;
  dg.bits  = bits;
  dg.shift = 0;
  for (int j = 0; j < i; ++j) dg.shift += bits / passes + (j < bits % passes ? 1 : 0);
  dg.width = bits / passes + (i < bits % passes ? 1 : 0);
  return dg;
}

int tiles_of(int64_t n) { return static_cast<int>(std::max<int64_t>((n + kTileRows - 1) / kTileRows, 1)); }

// *total = offsets[items - 1] + counts[items - 1]: the rows of an exclusive scan.
__global__ void k_radix_total(const uint32_t* counts, const uint32_t* offsets, int items, uint32_t* total)
{
  *total = offsets[items - 1] + counts[items - 1];
}

// Whether the first pass can read the caller's columns as raw runs of bytes
// (a single plain 8-byte key column without nulls -- its bits are the packed
// key -- and value columns without dictionaries); `src` then points at them,
// each pointer advanced by its column's offset.
// The caller's key column when it is a single plain 8-byte column without
// nulls (its bits are the packed key), advanced by its offset; else nullptr.
const uint64_t* plain_key_column(const Plan& p)
{
  const KeyCol& kc = p.key.cols[0];
  if (p.key.nwords != 1 || p.key.ncols != 1 || kc.width != 8 || kc.is_float || kc.is_bool || kc.null_bit ||
      kc.mask != nullptr || kc.shift != 0)
    return nullptr;
  return reinterpret_cast<const uint64_t*>(static_cast<const unsigned char*>(kc.data) + kc.offset * 8);
}

bool first_pass_columns(const Plan& p, const PartBufs& out, PartBufs& src)
{
  const uint64_t* key = plain_key_column(p);
  if (key == nullptr) return false;
  src         = PartBufs{};
  src.keys[0] = key;
  for (int c = 0; c < p.nchan; ++c) {
    const Channel& ch = p.chan[c];
    if (ch.dict_data != nullptr) return false;
    src.col[c].width = out.col[c].width;
    src.col[c].vals  = static_cast<const unsigned char*>(ch.data) + ch.offset * out.col[c].width;
  }
  return true;
}

// One pass; the first (FROM_COLUMNS) writes the rows it keeps to *n_active,
// which the later passes read.
template <int NW, bool FROM_COLUMNS>
cudaError_t radix_pass(const Plan& p, const PartBufs& in, int64_t n, uint32_t* n_active, const Digit& dg,
                       int ntiles, uint32_t* counts, uint32_t* offsets, void* temp, size_t temp_bytes,
                       const PartBufs& out, int32_t* status, bool hist_done, cudaStream_t st)
{
  cudaError_t e;
  if (!hist_done) {
    k_radix_hist<NW, FROM_COLUMNS><<<ntiles, kRadixBlock, 0, st>>>(p, in, n, n_active, dg, ntiles, counts, nullptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  const int items = ntiles << dg.width;
  e = scan_exclusive_u32(counts, offsets, items, temp, &temp_bytes, st);
  if (e != cudaSuccess) return e;
  if constexpr (FROM_COLUMNS) {
    // rows kept by the first pass: the later passes' row count
    k_radix_total<<<1, 1, 0, st>>>(counts, offsets, items, n_active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  PartBufs user{};
  const bool bulk_first = FROM_COLUMNS && first_pass_columns(p, out, user);
  if (!FROM_COLUMNS || bulk_first) {
    e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_radix_scatter_bulk<NW>), kBulkSmem);
    if (e != cudaSuccess) return e;
    k_radix_scatter_bulk<NW><<<ntiles, kRadixBlock, kBulkSmem, st>>>(p, bulk_first ? user : in, n_active, n,
                                                                     bulk_first, dg, offsets, ntiles, out, status);
  } else {
    e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_radix_scatter<NW>), kScatterSmem);
    if (e != cudaSuccess) return e;
    k_radix_scatter<NW><<<ntiles, kRadixBlock, kScatterSmem, st>>>(p, in, n, n_active, dg, ntiles, offsets, out, status);
  }
  return cudaGetLastError();
}

template <int NW>
cudaError_t radix_all(const Plan& p, int64_t n, int bits, uint32_t* n_active, const PartBufs& dst,
                      const PartBufs& tmp, uint32_t* counts, uint32_t* offsets, void* temp, size_t temp_bytes,
                      int32_t* status, bool hist0_done, cudaStream_t st)
{
  const int passes     = (bits + 7) / 8;
  const int ntiles     = tiles_of(n);
  const PartBufs* prev = nullptr;
  for (int i = 0; i < passes; ++i) {
    const Digit dg = pass_digit(bits, i);
    // the last pass writes `dst`; earlier ones alternate so that it does
    const PartBufs& out = ((passes - 1 - i) % 2 == 0) ? dst : tmp;
    cudaError_t e;
    if (i == 0)
      e = radix_pass<NW, true>(p, out, n, n_active, dg, ntiles, counts, offsets, temp, temp_bytes, out, status,
                               hist0_done, st);
    else
      e = radix_pass<NW, false>(p, *prev, n, n_active, dg, ntiles, counts, offsets, temp, temp_bytes, out, status,
                                false, st);
    if (e != cudaSuccess) return e;
    prev = &out;
  }
  return cudaSuccess;
}
}  // namespace

cudaError_t launch_part_radix_hist0(const Plan& p, int64_t n, int bits, uint32_t* counts, uint32_t* bucket_counts,
                                    cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  const Digit dg   = pass_digit(bits, 0);
  const int ntiles = tiles_of(n);
  const PartBufs none{};
  if (const uint64_t* key = plain_key_column(p)) {
    // the key column read as it lies (no per-row key packing)
    PartBufs src{};
    src.keys[0] = key;
    k_radix_hist<1, true, true><<<ntiles, kRadixBlock, 0, st>>>(p, src, n, nullptr, dg, ntiles, counts, bucket_counts);
  } else if (p.key.nwords == 1)
    k_radix_hist<1, true><<<ntiles, kRadixBlock, 0, st>>>(p, none, n, nullptr, dg, ntiles, counts, bucket_counts);
  else
    k_radix_hist<2, true><<<ntiles, kRadixBlock, 0, st>>>(p, none, n, nullptr, dg, ntiles, counts, bucket_counts);
  return cudaGetLastError();
}

cudaError_t launch_part_radix(const Plan& p, int64_t n, int bits, uint32_t* n_kept, const PartBufs& dst,
                              const PartBufs& tmp, uint32_t* counts, uint32_t* offsets, void* temp,
                              size_t temp_bytes, int32_t* status, bool hist0_done, cudaStream_t st)
{
  if (n <= 0) return cudaMemsetAsync(n_kept, 0, sizeof(uint32_t), st);
  return p.key.nwords == 1
           ? radix_all<1>(p, n, bits, n_kept, dst, tmp, counts, offsets, temp, temp_bytes, status, hist0_done, st)
           : radix_all<2>(p, n, bits, n_kept, dst, tmp, counts, offsets, temp, temp_bytes, status, hist0_done, st);
}

}  // namespace gbx
