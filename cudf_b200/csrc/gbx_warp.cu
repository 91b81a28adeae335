// gbx_warp.cu -- warp-private shared-memory aggregation (low cardinality).
//
// Each warp owns a private open-addressing table in shared memory, so no other
// thread ever touches its slots: batches of 32 rows are deduplicated inside
// the warp and each slot is updated once per batch with plain loads and stores
// (gbx_warpcore.cuh).  This replaces the reference's per-row global atomics
// (hash/groupby_kernels.cuh:98-105, detail/aggregation/aggregation.cuh:558-573)
// and avoids 64-bit shared-memory atomics, which run at ~1.5 op/clk/SM on B200
// against ~8.5 for 32-bit ones.  At the end each warp merges its table into
// the global table (one set of red.global per occupied slot).
#include <algorithm>

#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

// blockDim.x / 32 private tables of sl.slots + 1 slots (sl.total bytes each),
// back to back in dynamic shared memory.  Warp w of the grid aggregates rows
// [w * rows_per_warp, (w + 1) * rows_per_warp).
template <int NW, int NCH>
__global__ void __launch_bounds__(256, 2) k_agg_warp(const __grid_constant__ Plan plan,
                                                  const __grid_constant__ TableRef t,
                                                  const __grid_constant__ SmemLayout sl,
                                                  int64_t n,
                                                  int64_t rows_per_warp,
                                                  uint32_t max_probes)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  WarpTable<NW> T{smem + static_cast<size_t>(warp) * sl.total, &sl, sl.slots};
  T.reset(plan.acc, lane);

  const RowSource src{&plan};
  const Level<Global> G = global_level(t);
  const int64_t wid     = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
  const int64_t begin   = wid * rows_per_warp;
  const int64_t end     = min(n, begin + rows_per_warp);
  bool special          = false;  // warp-uniform: the reserved slot is in use

  // software pipeline: the next batch's keys and values load while this one
  // is probed and applied
  int64_t r       = begin + lane;
  uint64_t k[NW];
  bool act        = (r < end) && src.key<NW>(r, k);
  RowVals<NCH> v;
  load_row_values(plan, src, act, r, v, t.status);
  for (int64_t base = begin; base < end; base += 32) {
    const int64_t rn = base + 32 + lane;
    uint64_t kn[NW];
    const bool actn = (rn < end) && src.key<NW>(rn, kn);
    RowVals<NCH> vn;
    load_row_values(plan, src, actn, rn, vn, t.status);

    uint32_t slot;
    const int state = warp_find_or_insert<NW>(T, plan.acc, act, k, lane, slot);
    if (__any_sync(kFull, state == ST_FOUND && slot == T.S)) special = true;
    if (state == ST_SPILL) {
      int64_t g = global_slot<NW>(t, k, max_probes);
      if (g >= 0) accumulate_row<Global>(plan, G, g, r, t.status);
    }
    warp_accumulate(plan, T.tb, sl, state == ST_FOUND, slot, v, lane);

    r   = rn;
    act = actn;
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = kn[w];
    v = vn;
  }

  // merge the private table into the global one
  const Level<Shared> L{static_cast<uint32_t>(__cvta_generic_to_shared(T.tb)), &sl};
  const uint64_t* keys = T.keys();
  for (uint32_t s = lane; s <= T.S; s += 32) {
    uint64_t k[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = keys[s * NW + w];
    const bool occupied = (s < T.S) ? !key_is_empty<NW>(k) : special;
    if (!occupied) continue;
    int64_t g = global_slot<NW>(t, k, max_probes);
    if (g >= 0) merge_slot<Shared>(plan, L, s, G, g, t.status);
  }
}

namespace {
template <int NW, int NCH>
cudaError_t launch_agg_warp_impl(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                                 uint32_t max_probes, cudaStream_t st)
{
  const int block   = 256;
  const int warps   = block / 32;
  const size_t smem = static_cast<size_t>(sl.total) * warps;
  cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_agg_warp<NW, NCH>), smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e          = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_agg_warp<NW, NCH>, block, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int64_t grid = static_cast<int64_t>(num_sms) * per_sm;
  // at least 4 batches of 32 rows per warp
  const int64_t max_grid = (n + static_cast<int64_t>(warps) * 128 - 1) / (static_cast<int64_t>(warps) * 128);
  grid                   = std::max<int64_t>(1, std::min<int64_t>(grid, max_grid));
  int64_t rpw            = (n + grid * warps - 1) / (grid * warps);
  rpw                    = (rpw + 31) / 32 * 32;
  k_agg_warp<NW, NCH><<<static_cast<int>(grid), block, smem, st>>>(p, t, sl, n, rpw, max_probes);
  return cudaGetLastError();
}

template <int NW>
cudaError_t launch_agg_warp_nw(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                               uint32_t max_probes, cudaStream_t st)
{
  if (p.nchan <= 2) return launch_agg_warp_impl<NW, 2>(p, t, sl, n, num_sms, max_probes, st);
  if (p.nchan <= 4) return launch_agg_warp_impl<NW, 4>(p, t, sl, n, num_sms, max_probes, st);
  return launch_agg_warp_impl<NW, kMaxChannels>(p, t, sl, n, num_sms, max_probes, st);
}
}  // namespace

cudaError_t launch_agg_warp(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                            uint32_t max_probes, cudaStream_t st)
{
  return p.key.nwords == 1 ? launch_agg_warp_nw<1>(p, t, sl, n, num_sms, max_probes, st)
                           : launch_agg_warp_nw<2>(p, t, sl, n, num_sms, max_probes, st);
}

}  // namespace gbx
