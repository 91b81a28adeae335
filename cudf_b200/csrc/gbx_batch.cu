// gbx_batch.cu -- kernels of the batched groupby (gbx_batch.hpp).
//
// A libcudf caller with many small tables runs one groupby per table:
// cudf::groupby::groupby(keys_i).aggregate(requests_i) (groupby.cu:197-221),
// each with its own set build, aggregation pass, compaction, gathers and
// result-size synchronisation (hash/groupby.cu:548-622).  Here all instances
// go through one persistent kernel: CTAs claim (instance, row range) items
// from a counter and aggregate each with the instance's mode -- a CTA-shared
// table (the privatised kernel's scheme), a table per warp (the warp core's
// scheme), or direct global updates -- into the instance's own global table.
// Counting, scanning and writing the groups of all instances then take three
// more launches, so the whole batch is one CUDA graph.
#include <cuda_runtime.h>

#include "gbx_batch.hpp"
#include "gbx_scan.hpp"
#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {

// ------------------------------------------------------------ row source

// Key buffers of one instance (layout from the schema's KeyPlan).
struct InstKeyBufs {
  const InstCols* ic;
  __device__ __forceinline__ const void* data(int c) const { return ic->key[c].data; }
  __device__ __forceinline__ const uint32_t* mask(int c) const { return ic->key[c].mask; }
  __device__ __forceinline__ int64_t offset(int c) const { return ic->key[c].offset; }
};

// Rows of one instance: the schema plan gives element layouts, the
// instance's InstCols the buffers.
struct BatchSource {
  const Plan* plan;
  const InstCols* ic;
  template <int NW>
  __device__ __forceinline__ bool key(int64_t r, uint64_t (&k)[NW]) const
  {
    return pack_key_from<NW>(plan->key, InstKeyBufs{ic}, r, k);
  }
  __device__ __forceinline__ bool value(int c, int64_t r, uint64_t& b, int32_t* status) const
  {
    const InstChan& ch = ic->chan[c];
    if (!bit_valid(ch.mask, r + ch.offset)) return false;
    bool ok;
    b = value_bits_at(plan->chan[c], ch.data, ch.offset, ch.dict_data, ch.dict_offset, ch.dict_size, r, ok);
    if (!ok) {
      atomicOr(status, S_BAD_INDEX);
      return false;
    }
    return true;
  }
};

__device__ __forceinline__ uint32_t probe_limit(uint64_t cap) { return static_cast<uint32_t>(cap < 4096 ? cap : 4096); }

// A row whose value bits were loaded ahead (RowVals), read through the
// row-source interface of accumulate_row_from.
template <int NCH>
struct LoadedRow {
  const RowVals<NCH>* v;
  __device__ __forceinline__ bool value(int c, int64_t, uint64_t& b, int32_t*) const
  {
    // selected with constant indices, so that the values stay in registers
    b = 0;
#pragma unroll
    for (int i = 0; i < NCH; ++i)
      if (i == c) b = v->bits[i];
    return (v->valid >> c) & 1u;
  }
};


// --------------------------------------------------------- per-item modes

// CTA-shared table with shared-memory atomics; rows whose key finds no room
// go to the global table; the table is merged into the global one at the end.
template <int NW, int NCH, int BLOCK>
__device__ __forceinline__ void item_shared(const Plan& plan, const BatchInst& I, unsigned char* smem,
                                            uint32_t& s_special, int64_t begin, int64_t end)
{
  const SmemLayout& sl = I.sl;
  const uint32_t S     = sl.slots;
  const uint32_t base  = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  uint64_t* skeys      = reinterpret_cast<uint64_t*>(smem + sl.keys_off);
  uint32_t* srows      = reinterpret_cast<uint32_t*>(smem + sl.rows_off);
  for (uint32_t s = threadIdx.x; s <= S; s += BLOCK) {
#pragma unroll
    for (int w = 0; w < NW; ++w) skeys[s * NW + w] = kEmptyWord;
    srows[s] = 0;
    for (int a = 0; a < plan.acc.nacc; ++a) {
      const uint64_t id = identity_bits(plan.acc.kind[a]);
      if (acc_bytes(plan.acc.kind[a]) == 4) reinterpret_cast<uint32_t*>(smem + sl.acc_off[a])[s] = static_cast<uint32_t>(id);
      else reinterpret_cast<uint64_t*>(smem + sl.acc_off[a])[s] = id;
    }
  }
  __syncthreads();

  const BatchSource src{&plan, &I.cols};
  const Level<Shared> L{base, &sl};
  const Level<Global> G{&I.t};
  const uint32_t keys        = base + sl.keys_off;
  const uint32_t smem_probes = S < 32 ? S : 32;
  const uint32_t max_probes  = probe_limit(I.t.cap);
  // the next row's key and values load while this row is applied
  int64_t r = begin + threadIdx.x;
  uint64_t k[NW];
  bool act = r < end && src.key<NW>(r, k);
  RowVals<NCH> v;
  load_row_values(plan, src, act, r, v, I.t.status);
  for (; r < end; r += BLOCK) {
    const int64_t rn = r + BLOCK;
    uint64_t kn[NW];
    const bool actn = rn < end && src.key<NW>(rn, kn);
    RowVals<NCH> vn;
    load_row_values(plan, src, actn, rn, vn, I.t.status);
    if (act) {
      int64_t s;
      if (key_is_empty<NW>(k)) {
        s = S;
        if (s_special == 0) s_special = 1;
      } else {
        s = find_or_insert<Shared, NW>(keys, S - 1, k, hash_key<NW>(k), smem_probes);
      }
      const LoadedRow<NCH> lr{&v};
      if (s >= 0) {
        accumulate_row_from<Shared>(plan, lr, L, s, r, I.t.status);
      } else {
        const int64_t g = global_slot<NW>(I.t, k, max_probes);
        if (g >= 0) accumulate_row_from<Global>(plan, lr, G, g, r, I.t.status);
      }
    }
    act = actn;
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = kn[w];
    v = vn;
  }
  __syncthreads();

  for (uint32_t s = threadIdx.x; s <= S; s += BLOCK) {
    uint64_t k[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = skeys[s * NW + w];
    const bool occupied = (s < S) ? !key_is_empty<NW>(k) : (s_special != 0);
    if (!occupied) continue;
    const int64_t g = global_slot<NW>(I.t, k, max_probes);
    if (g >= 0) merge_slot<Shared>(plan, L, s, G, g, I.t.status);
  }
}

// A shared-memory table per warp, updated without atomics (gbx_warpcore.cuh);
// the item's rows are split into one contiguous run per warp.
template <int NW, int NCH, int BLOCK>
__device__ __forceinline__ void item_warp(const Plan& plan, const BatchInst& I, unsigned char* smem, int64_t begin,
                                          int64_t end)
{
  constexpr int kWarps = BLOCK / 32;
  const int lane       = threadIdx.x & 31;
  const int warp       = threadIdx.x >> 5;
  const SmemLayout& sl = I.sl;
  WarpTable<NW> T{smem + static_cast<size_t>(warp) * sl.total, &sl, sl.slots};
  T.reset(plan.acc, lane);

  const BatchSource src{&plan, &I.cols};
  const Level<Global> G{&I.t};
  const uint32_t max_probes = probe_limit(I.t.cap);
  int64_t chunk             = (end - begin + kWarps - 1) / kWarps;
  chunk                     = (chunk + 31) & ~int64_t(31);
  const int64_t wb          = begin + warp * chunk;
  const int64_t we          = min(end, wb + chunk);
  bool special              = false;

  int64_t r = wb + lane;
  uint64_t k[NW];
  bool act = (r < we) && src.key<NW>(r, k);
  RowVals<NCH> v;
  load_row_values(plan, src, act, r, v, I.t.status);
  for (int64_t b = wb; b < we; b += 32) {
    const int64_t rn = b + 32 + lane;
    uint64_t kn[NW];
    const bool actn = (rn < we) && src.key<NW>(rn, kn);
    RowVals<NCH> vn;
    load_row_values(plan, src, actn, rn, vn, I.t.status);

    uint32_t slot;
    const int state = warp_find_or_insert<NW>(T, plan.acc, act, k, lane, slot);
    if (__any_sync(kFull, state == ST_FOUND && slot == T.S)) special = true;
    if (state == ST_SPILL) {
      const int64_t g = global_slot<NW>(I.t, k, max_probes);
      if (g >= 0) accumulate_row_from<Global>(plan, src, G, g, r, I.t.status);
    }
    warp_accumulate(plan, T.tb, sl, state == ST_FOUND, slot, v, lane);

    r   = rn;
    act = actn;
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = kn[w];
    v = vn;
  }

  const Level<Shared> L{static_cast<uint32_t>(__cvta_generic_to_shared(T.tb)), &sl};
  const uint64_t* keys = T.keys();
  for (uint32_t s = lane; s <= T.S; s += 32) {
    uint64_t kk[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) kk[w] = keys[s * NW + w];
    const bool occupied = (s < T.S) ? !key_is_empty<NW>(kk) : special;
    if (!occupied) continue;
    const int64_t g = global_slot<NW>(I.t, kk, max_probes);
    if (g >= 0) merge_slot<Shared>(plan, L, s, G, g, I.t.status);
  }
}

// Every row updates the instance's global table.
template <int NW, int NCH, int BLOCK>
__device__ __forceinline__ void item_global(const Plan& plan, const BatchInst& I, int64_t begin, int64_t end)
{
  const BatchSource src{&plan, &I.cols};
  const Level<Global> G{&I.t};
  const uint32_t max_probes = probe_limit(I.t.cap);
  int64_t r = begin + threadIdx.x;
  uint64_t k[NW];
  bool act = r < end && src.key<NW>(r, k);
  RowVals<NCH> v;
  load_row_values(plan, src, act, r, v, I.t.status);
  for (; r < end; r += BLOCK) {
    const int64_t rn = r + BLOCK;
    uint64_t kn[NW];
    const bool actn = rn < end && src.key<NW>(rn, kn);
    RowVals<NCH> vn;
    load_row_values(plan, src, actn, rn, vn, I.t.status);
    if (act) {
      const int64_t g = global_slot<NW>(I.t, k, max_probes);
      if (g >= 0) accumulate_row_from<Global>(plan, LoadedRow<NCH>{&v}, G, g, r, I.t.status);
    }
    act = actn;
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = kn[w];
    v = vn;
  }
}

// ---------------------------------------------------------------- kernels

template <int NW, int NCH, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK) k_batch_agg(const __grid_constant__ Plan plan,
                                                                  const BatchInst* __restrict__ insts,
                                                                  const BatchItem* __restrict__ items,
                                                                  uint32_t nitems,
                                                                  uint32_t* counter)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchInst s_inst;
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_special;
  static_assert(sizeof(BatchInst) % 16 == 0, "BatchInst is copied as 16-byte vectors");

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t it = s_item;
    if (it >= nitems) break;
    const BatchItem item = items[it];
    {
      const uint4* src = reinterpret_cast<const uint4*>(insts + item.inst);
      uint4* dst       = reinterpret_cast<uint4*>(&s_inst);
      for (int i = threadIdx.x; i < static_cast<int>(sizeof(BatchInst) / 16); i += BLOCK) dst[i] = __ldg(src + i);
    }
    if (threadIdx.x == 0) s_special = 0;
    __syncthreads();
    switch (s_inst.mode) {
      case BM_SHARED: item_shared<NW, NCH, BLOCK>(plan, s_inst, smem, s_special, item.begin, item.end); break;
      case BM_WARP: item_warp<NW, NCH, BLOCK>(plan, s_inst, smem, item.begin, item.end); break;
      default: item_global<NW, NCH, BLOCK>(plan, s_inst, item.begin, item.end); break;
    }
    __syncthreads();  // s_inst and the shared tables are rewritten by the next item
  }
}

// Sampled distinct count per instance: one CTA per instance inserts up to
// `per_inst` evenly spaced rows' hashes into a shared-memory set.
constexpr int kSampleSet = 4096;

template <int NW>
__global__ void __launch_bounds__(256) k_batch_sample(const __grid_constant__ Plan plan,
                                                      const BatchInst* __restrict__ insts, int ninst, int per_inst,
                                                      uint32_t* out)
{
  __shared__ uint64_t set[kSampleSet];
  __shared__ uint32_t counts[2];
  for (int i = blockIdx.x; i < ninst; i += gridDim.x) {
    for (int s = threadIdx.x; s < kSampleSet; s += blockDim.x) set[s] = kEmptyWord;
    if (threadIdx.x < 2) counts[threadIdx.x] = 0;
    __syncthreads();
    const BatchInst& I = insts[i];
    const int64_t n    = I.num_rows;
    const int64_t m    = n < per_inst ? n : per_inst;
    const BatchSource src{&plan, &I.cols};
    for (int64_t j = threadIdx.x; j < m; j += blockDim.x) {
      int64_t r = static_cast<int64_t>((static_cast<double>(j) + 0.5) * static_cast<double>(n) / static_cast<double>(m));
      if (r >= n) r = n - 1;
      uint64_t k[NW];
      if (!src.key<NW>(r, k)) continue;
      atomicAdd(&counts[0], 1u);
      uint64_t f = hash_key<NW>(k);
      if (f == kEmptyWord) f = 0;
      uint32_t s = static_cast<uint32_t>(fmix64(f ^ 0x5bd1e995ULL)) & (kSampleSet - 1);
      for (int p = 0; p < kSampleSet; ++p) {
        const unsigned long long old =
          atomicCAS(reinterpret_cast<unsigned long long*>(set + s), kEmptyWord, static_cast<unsigned long long>(f));
        if (old == kEmptyWord) {
          atomicAdd(&counts[1], 1u);
          break;
        }
        if (old == f) break;
        s = (s + 1) & (kSampleSet - 1);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      out[2 * i]     = counts[0];
      out[2 * i + 1] = counts[1];
    }
    __syncthreads();
  }
}

// Identity fill of every instance's global table (one CTA per instance).
template <int NW>
__global__ void __launch_bounds__(256) k_batch_init(const __grid_constant__ Plan plan,
                                                    const BatchInst* __restrict__ insts, int ninst)
{
  for (int i = blockIdx.x; i < ninst; i += gridDim.x) {
    const TableRef& t = insts[i].t;
    const uint64_t n  = t.cap + 1;
    for (uint64_t s = threadIdx.x; s < n; s += blockDim.x) {
#pragma unroll
      for (int w = 0; w < NW; ++w) t.keys[s * NW + w] = kEmptyWord;
      t.rows[s] = 0;
      for (int a = 0; a < plan.acc.nacc; ++a) {
        const uint64_t id = identity_bits(plan.acc.kind[a]);
        if (acc_bytes(plan.acc.kind[a]) == 4) reinterpret_cast<uint32_t*>(t.acc[a])[s] = static_cast<uint32_t>(id);
        else reinterpret_cast<uint64_t*>(t.acc[a])[s] = id;
      }
    }
    if (threadIdx.x == 0) {
      *t.special_used = 0;
      *t.status       = 0;
    }
  }
}

template <int NW>
__device__ __forceinline__ bool slot_occupied(const TableRef& t, uint64_t s)
{
  if (s == t.cap) return *t.special_used != 0;
  if constexpr (NW == 1) {
    return t.keys[s] != kEmptyWord;
  } else {
    return !(t.keys[2 * s] == kEmptyWord && t.keys[2 * s + 1] == kEmptyWord);
  }
}

// Position of the n-th (0-based) set bit of m, which has more than n set bits.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int n)
{
  int lo = 0, hi = 31;
  while (lo < hi) {
    const int mid        = (lo + hi) >> 1;
    const uint32_t below = (mid == 31) ? m : (m & ((2u << mid) - 1u));
    if (__popc(below) > n) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Occupied slots per instance (one CTA per instance).
template <int NW>
__global__ void __launch_bounds__(256) k_batch_count(const BatchInst* __restrict__ insts, int ninst, int64_t* counts)
{
  __shared__ unsigned long long total;
  for (int i = blockIdx.x; i < ninst; i += gridDim.x) {
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    const TableRef& t = insts[i].t;
    uint32_t local    = 0;
    for (uint64_t s = threadIdx.x; s <= t.cap; s += blockDim.x) local += slot_occupied<NW>(t, s) ? 1u : 0u;
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(kFull, local, off);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(&total, static_cast<unsigned long long>(local));
    __syncthreads();
    if (threadIdx.x == 0) counts[i] = static_cast<int64_t>(total);
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) counts[ninst] = 0;
}

// Output rows of every instance's groups (one CTA per instance): each warp
// takes 32 slots at a time, packs the occupied ones into a prefix of lanes
// and reserves that many rows of the instance's run.
template <int NW>
__global__ void __launch_bounds__(256) k_batch_write(const __grid_constant__ Plan plan,
                                                     const BatchInst* __restrict__ insts, int ninst,
                                                     const int64_t* __restrict__ offsets,
                                                     const __grid_constant__ OutPlan op)
{
  __shared__ uint32_t cursor;
  const int lane = threadIdx.x & 31;
  for (int i = blockIdx.x; i < ninst; i += gridDim.x) {
    if (threadIdx.x == 0) cursor = 0;
    __syncthreads();
    const TableRef& t    = insts[i].t;
    const int64_t out0   = offsets[i];
    const GlobalAccs A{&t};
    const uint64_t nslot = t.cap + 1;
    for (uint64_t b = threadIdx.x & ~31u; b < nslot; b += blockDim.x) {
      const uint64_t s   = b + lane;
      const bool occ     = s < nslot && slot_occupied<NW>(t, s);
      const uint32_t bal = __ballot_sync(kFull, occ);
      if (bal == 0) continue;
      const int cnt = __popc(bal);
      uint32_t pos  = 0;
      if (lane == 0) pos = atomicAdd(&cursor, static_cast<uint32_t>(cnt));
      pos = __shfl_sync(kFull, pos, 0);
      // lane j < cnt takes the j-th occupied slot of this chunk
      const bool active  = lane < cnt;
      const int src_lane = active ? nth_set_bit(bal, lane) : 0;
      const uint64_t my  = __shfl_sync(kFull, s, src_lane);
      uint64_t k[2]      = {0, 0};
      if (active) {
        if (my == t.cap) {
          k[0] = k[1] = kEmptyWord;
        } else {
#pragma unroll
          for (int w = 0; w < NW; ++w) k[w] = t.keys[my * NW + w];
        }
      }
      warp_write_groups(plan, op, A, active, my, k, out0 + pos, lane);
    }
    __syncthreads();
  }
}

inline int instance_grid(int ninst) { return ninst < 8192 ? (ninst > 0 ? ninst : 1) : 8192; }

// The launch sets no attribute (it may be recorded into a graph);
// batch_agg_max_grid, called before, raises the kernel's limit.
template <int NW, int NCH, int BLOCK>
struct AggF {
  static cudaError_t run(const Plan& p, const BatchInst* insts, const BatchItem* items, uint32_t nitems,
                         uint32_t* counter, int grid, size_t smem, cudaStream_t st)
  {
    if (smem > kBatchMaxDynamicSmem) return cudaErrorInvalidValue;
    k_batch_agg<NW, NCH, BLOCK><<<grid, BLOCK, smem, st>>>(p, insts, items, nitems, counter);
    return cudaGetLastError();
  }
};

template <int NW, int NCH, int BLOCK>
struct GridF {
  static cudaError_t run(size_t smem, int num_sms, int* grid)
  {
    if (smem > kBatchMaxDynamicSmem) return cudaErrorInvalidValue;
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_batch_agg<NW, NCH, BLOCK>), kBatchMaxDynamicSmem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_agg<NW, NCH, BLOCK>, BLOCK, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *grid = per_sm * num_sms;
    return cudaSuccess;
  }
};

// Dispatch over (key words, channel bound, block size).
template <template <int, int, int> class F, class... Args>
cudaError_t dispatch(const Plan& p, int block, Args&&... args)
{
  const bool nw1 = p.key.nwords == 1;
  const bool c2  = p.nchan <= 2;
  if (block == 512) {
    if (nw1) return c2 ? F<1, 2, 512>::run(args...) : F<1, kMaxChannels, 512>::run(args...);
    return c2 ? F<2, 2, 512>::run(args...) : F<2, kMaxChannels, 512>::run(args...);
  }
  if (nw1) return c2 ? F<1, 2, 256>::run(args...) : F<1, kMaxChannels, 256>::run(args...);
  return c2 ? F<2, 2, 256>::run(args...) : F<2, kMaxChannels, 256>::run(args...);
}

}  // namespace

cudaError_t launch_batch_sample(const Plan& schema, const BatchInst* insts, int ninst, int per_inst, uint32_t* out,
                                cudaStream_t st)
{
  if (ninst <= 0) return cudaSuccess;
  if (schema.key.nwords == 1) k_batch_sample<1><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst, per_inst, out);
  else k_batch_sample<2><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst, per_inst, out);
  return cudaGetLastError();
}

cudaError_t launch_batch_init(const Plan& schema, const BatchInst* insts, int ninst, cudaStream_t st)
{
  if (ninst <= 0) return cudaSuccess;
  if (schema.key.nwords == 1) k_batch_init<1><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst);
  else k_batch_init<2><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst);
  return cudaGetLastError();
}

cudaError_t launch_batch_agg(const Plan& schema, const BatchInst* insts, const BatchItem* items, uint32_t nitems,
                             uint32_t* counter, int block, int grid, size_t smem, cudaStream_t st)
{
  if (nitems == 0) return cudaSuccess;
  return dispatch<AggF>(schema, block, schema, insts, items, nitems, counter, grid, smem, st);
}

cudaError_t batch_agg_max_grid(const Plan& schema, int block, size_t smem, int num_sms, int* grid)
{
  return dispatch<GridF>(schema, block, smem, num_sms, grid);
}

cudaError_t launch_batch_count(const Plan& schema, const BatchInst* insts, int ninst, int64_t* counts,
                               int64_t* offsets, void* temp, size_t* temp_bytes, cudaStream_t st)
{
  if (temp == nullptr) return scan_exclusive_i64(nullptr, nullptr, ninst + 1, nullptr, temp_bytes, st);
  if (schema.key.nwords == 1) k_batch_count<1><<<instance_grid(ninst), 256, 0, st>>>(insts, ninst, counts);
  else k_batch_count<2><<<instance_grid(ninst), 256, 0, st>>>(insts, ninst, counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return scan_exclusive_i64(counts, offsets, ninst + 1, temp, temp_bytes, st);
}

cudaError_t launch_batch_write(const Plan& schema, const BatchInst* insts, int ninst, const int64_t* offsets,
                               const OutPlan& op, cudaStream_t st)
{
  if (ninst <= 0) return cudaSuccess;
  if (schema.key.nwords == 1) k_batch_write<1><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst, offsets, op);
  else k_batch_write<2><<<instance_grid(ninst), 256, 0, st>>>(schema, insts, ninst, offsets, op);
  return cudaGetLastError();
}

}  // namespace gbx
