// gbx_tiled.cu -- low-cardinality aggregation by grouping each tile of rows
// before touching the table.
//
// With few groups (up to ~500) every CTA holds the whole group table in shared
// memory.  Applying each row to it costs ~13 shared-memory atomics per row for
// the 100M-row workload's 12 accumulators, and the 64-bit ones run as
// compare-and-swap loops that conflict when many lanes hit the same few slots:
// the per-row atomic path measured 35.7 warp-instructions per row on B200.
// Here a CTA instead takes up to 4,096 rows at a time and
//   1. loads the tile's keys and, per channel, its values and validity into
//      shared memory (coalesced, every load of a batch in flight together),
//      then finds each row's slot in its table and takes the next rank of that
//      slot with one 32-bit shared atomic;
//   2. scans the slot counts and lists the tile's rows group by group;
//   3. folds each group's rows in one thread's registers (ChanAcc), reading the
//      staged values, then merges that into the group's slot with plain
//      read-modify-writes -- the thread owns the slot for the step, so no
//      atomics are needed.
// A group with r rows in the tile updates its slot once instead of r times.
// Rows whose key finds no room in the table go to the global table directly,
// and every CTA merges its table into the global one at the end, as the
// per-CTA privatised kernel does (the reference's shared-memory aggregation,
// hash/groupby.cu:424-504, restated with tile-local grouping).
#include <cub/block/block_scan.cuh>

#include <algorithm>

#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kTiledBlock    = 512;
constexpr int kTiledPer      = 8;  // at most this many rows per thread per tile
constexpr int kTiledMaxRows  = kTiledBlock * kTiledPer;
constexpr int kTiledMaxSlots = 1024;
constexpr int kScanPer       = (kTiledMaxSlots + 1 + kTiledBlock - 1) / kTiledBlock;
constexpr uint32_t kNoRec    = 0xffffffffu;
constexpr int kChunk         = 16;  // rows of one group folded by one thread
// chunks of one tile: sum over groups of ceil(rows / kChunk)
constexpr int kMaxChunks = kTiledMaxRows / kChunk + kTiledMaxSlots + 1;
// dynamic shared memory per CTA so that two CTAs fit an SM (228 KB, less
// 1 KB reserved and ~2 KB of static shared memory per CTA)
constexpr size_t kTiledSmemBudget = 110 * 1024;

// Folds `len` staged rows of one group (tile-local indices rows[0..len)) of a
// channel of physical type PT into A.
template <int PT>
__device__ __forceinline__ void fold_chunk(const Channel& ch, const uint64_t* cv, const uint8_t* cvv,
                                           const uint16_t* rows, uint32_t len, ChanAcc& A)
{
  const uint32_t roles = chan_roles(ch);
  for (uint32_t j = 0; j < len; ++j) {
    const uint32_t li = rows[j];
    if (cvv[li]) chan_acc_add<PT>(ch, roles, A, cv[li]);
  }
}

// Merges a chunk's accumulators into slot s of the CTA table with shared
// atomics (several chunks of a group merge at once).  The slot's shift was
// fixed before the chunks were folded, so A.s2 and A.s1 are relative to it.
__device__ __forceinline__ void merge_partial(const Channel& ch, const ChanAcc& A, const Level<Shared>& L, uint32_t s,
                                              int32_t* status)
{
  if (A.cnt == 0) return;
  if (ch.a_cnt >= 0) Shared::add_u32(L.acc(ch.a_cnt) + s * 4, A.cnt);
  const bool m64 = minmax_is64(ch.ptype);
  if (ch.a_min >= 0) {
    if (m64) Shared::min_u64(L.acc(ch.a_min) + s * 8, A.mn);
    else Shared::min_u32(L.acc(ch.a_min) + s * 4, static_cast<uint32_t>(A.mn));
  }
  if (ch.a_max >= 0) {
    if (m64) Shared::max_u64(L.acc(ch.a_max) + s * 8, A.mx);
    else Shared::max_u32(L.acc(ch.a_max) + s * 4, static_cast<uint32_t>(A.mx));
  }
  if (ch.is_float) {
    if (ch.a_sum >= 0) Shared::add_f64(L.acc(ch.a_sum) + s * 8, __longlong_as_double(static_cast<long long>(A.sum)));
    if (ch.a_sq >= 0) Shared::add_f64(L.acc(ch.a_sq) + s * 8, __longlong_as_double(static_cast<long long>(A.sq)));
    if (ch.a_prod >= 0)
      mul_cas_f64<Shared>(L.acc(ch.a_prod) + s * 8, __longlong_as_double(static_cast<long long>(A.prod)), status);
  } else {
    if (ch.a_sum >= 0) Shared::add_u64(L.acc(ch.a_sum) + s * 8, A.sum);
    if (ch.a_sq >= 0) Shared::add_u64(L.acc(ch.a_sq) + s * 8, A.sq);
    if (ch.a_prod >= 0) mul_cas_i64<Shared>(L.acc(ch.a_prod) + s * 8, static_cast<int64_t>(A.prod), status);
  }
  if (ch.a_k >= 0) Shared::add_f64(L.acc(ch.a_s2) + s * 8, A.s2);
  if (ch.a_s1 >= 0) Shared::add_f64(L.acc(ch.a_s1) + s * 8, A.s1);
}

// Byte offsets of the per-tile staging areas in dynamic shared memory, after
// the table: slot counts, first positions and first chunks ((S + 1) u32
// each), the slot of each chunk (u16), the tile's rows in group order (u16),
// each channel's value bits (u64) and validity bytes for tile_rows rows.
struct TiledLayout {
  uint32_t cnt_off, off_off, coff_off, cslot_off, perm_off, vals_off, valid_off, total;
  int tile_rows;
};

TiledLayout tiled_layout(const SmemLayout& sl, int nchan, int tile_rows)
{
  TiledLayout tl{};
  tl.tile_rows = tile_rows;
  uint32_t o   = sl.total;
  tl.cnt_off   = o;
  o += (sl.slots + 1) * 4;
  tl.off_off = o;
  o += (sl.slots + 1) * 4;
  tl.coff_off = o;
  o += (sl.slots + 1) * 4;
  tl.cslot_off = o;
  o += kMaxChunks * 2;
  tl.perm_off = o;
  o += tile_rows * 2;
  o           = (o + 7) & ~7u;
  tl.vals_off = o;
  o += static_cast<uint32_t>(nchan) * tile_rows * 8;
  tl.valid_off = o;
  o += static_cast<uint32_t>(nchan) * tile_rows;
  tl.total = (o + 15) & ~15u;
  return tl;
}

// The largest tile (a multiple of the block, at most kTiledMaxRows) whose
// staging fits kTiledSmemBudget; tile_rows 0 when none does.
TiledLayout pick_tiled_layout(const SmemLayout& sl, int nchan)
{
  for (int rows = kTiledMaxRows; rows >= kTiledBlock; rows -= kTiledBlock) {
    const TiledLayout tl = tiled_layout(sl, nchan, rows);
    if (tl.total <= kTiledSmemBudget) return tl;
  }
  TiledLayout none{};
  return none;
}

// PART: the rows are the bucket-ordered copies `pb` of the radix
// partitioning (*n_part of them) and each CTA takes one contiguous run of
// tiles, so that its table only sees the groups of the few buckets the run
// covers; otherwise the caller's n rows, tiles dealt round-robin.
template <int NW, bool PART>
__global__ void __launch_bounds__(kTiledBlock, 2) k_agg_tiled(const __grid_constant__ Plan plan,
                                                           const __grid_constant__ TableRef t,
                                                           const __grid_constant__ SmemLayout sl,
                                                           const __grid_constant__ TiledLayout tl, int64_t n,
                                                           const __grid_constant__ PartBufs pb,
                                                           const uint32_t* n_part, uint32_t smem_probes,
                                                           uint32_t max_probes)
{
  extern __shared__ __align__(16) unsigned char smem[];
  using BlockScan = cub::BlockScan<uint32_t, kTiledBlock>;
  __shared__ typename BlockScan::TempStorage scan_tmp;
  __shared__ uint32_t s_special;
  const uint32_t S     = sl.slots;
  const int tile_rows  = tl.tile_rows;
  const int per        = tile_rows / kTiledBlock;
  uint64_t* skeys      = reinterpret_cast<uint64_t*>(smem + sl.keys_off);
  uint32_t* srows      = reinterpret_cast<uint32_t*>(smem + sl.rows_off);
  uint32_t* cnt        = reinterpret_cast<uint32_t*>(smem + tl.cnt_off);
  uint32_t* off        = reinterpret_cast<uint32_t*>(smem + tl.off_off);
  uint32_t* coff       = reinterpret_cast<uint32_t*>(smem + tl.coff_off);
  uint16_t* cslot      = reinterpret_cast<uint16_t*>(smem + tl.cslot_off);
  uint16_t* perm       = reinterpret_cast<uint16_t*>(smem + tl.perm_off);
  uint64_t* vals       = reinterpret_cast<uint64_t*>(smem + tl.vals_off);
  uint8_t* valid       = smem + tl.valid_off;
  const uint32_t base  = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t keys  = base + sl.keys_off;

  // identity fill, counts zeroed
  for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) {
#pragma unroll
    for (int w = 0; w < NW; ++w) skeys[s * NW + w] = kEmptyWord;
    srows[s] = 0;
    cnt[s]   = 0;
    for (int a = 0; a < plan.acc.nacc; ++a) {
      const uint64_t id = identity_bits(plan.acc.kind[a]);
      if (acc_bytes(plan.acc.kind[a]) == 4) reinterpret_cast<uint32_t*>(smem + sl.acc_off[a])[s] = static_cast<uint32_t>(id);
      else reinterpret_cast<uint64_t*>(smem + sl.acc_off[a])[s] = id;
    }
  }
  if (threadIdx.x == 0) s_special = 0;
  __syncthreads();

  const Level<Global> G = global_level(t);
  const RowSource src{&plan};
  const PartSource psrc{&pb};
  if constexpr (PART) n = *n_part;
  const int64_t ntiles     = (n + tile_rows - 1) / tile_rows;
  const int64_t tile_begin = PART ? ntiles * blockIdx.x / gridDim.x : blockIdx.x;
  const int64_t tile_end   = PART ? ntiles * (blockIdx.x + 1) / gridDim.x : ntiles;
  const int64_t tile_step  = PART ? 1 : gridDim.x;
  for (int64_t tile = tile_begin; tile < tile_end; tile += tile_step) {
    const int64_t t0 = tile * tile_rows;
    // 1a. keys (this thread's rows threadIdx.x + q * kTiledBlock)
    uint64_t k[kTiledPer][NW];
    bool kept[kTiledPer];
#pragma unroll
    for (int q = 0; q < kTiledPer; ++q) {
      const int64_t r = t0 + threadIdx.x + q * kTiledBlock;
      if constexpr (PART) kept[q] = q < per && r < n && psrc.key<NW>(r, k[q]);
      else kept[q] = q < per && r < n && pack_key<NW>(plan.key, r, k[q]);
    }
    // 1b. values and validity of the kept rows, staged channel by channel
    for (int c = 0; c < plan.nchan; ++c) {
      const Channel& ch = plan.chan[c];
      uint64_t* cv      = vals + static_cast<size_t>(c) * tile_rows;
      uint8_t* cvv      = valid + static_cast<size_t>(c) * tile_rows;
      if constexpr (PART) {
        const PartCol& pc = pb.col[c];
        uint64_t b[kTiledPer];
        bool v[kTiledPer];
#pragma unroll
        for (int q = 0; q < kTiledPer; ++q) {
          const int64_t i = t0 + threadIdx.x + q * kTiledBlock;
          b[q]            = kept[q] ? load_bits(pc.vals, i, pc.width) : 0;
          v[q]            = kept[q] && (pc.valid == nullptr || __ldg(pc.valid + i) != 0);
        }
#pragma unroll
        for (int q = 0; q < kTiledPer; ++q) {
          if (!kept[q]) continue;
          const int li = threadIdx.x + q * kTiledBlock;
          cv[li]       = v[q] ? b[q] : 0;
          cvv[li]      = v[q] ? 1 : 0;
        }
      } else if (ch.dict_data == nullptr) {
        const int w = pt_width(ch.ptype);
        uint64_t b[kTiledPer];
        bool v[kTiledPer];
#pragma unroll
        for (int q = 0; q < kTiledPer; ++q) {
          const int64_t i = t0 + threadIdx.x + q * kTiledBlock + ch.offset;
          b[q]            = kept[q] ? load_bits(ch.data, i, w) : 0;
          v[q]            = kept[q] && bit_valid(ch.mask, i);
        }
#pragma unroll
        for (int q = 0; q < kTiledPer; ++q) {
          if (!kept[q]) continue;
          const int li = threadIdx.x + q * kTiledBlock;
          cv[li]       = v[q] ? b[q] : 0;
          cvv[li]      = v[q] ? 1 : 0;
        }
      } else {
        for (int q = 0; q < kTiledPer; ++q) {
          if (!kept[q]) continue;
          const int li = threadIdx.x + q * kTiledBlock;
          uint64_t b   = 0;
          const bool v = src.value(c, t0 + li, b, t.status);
          cv[li]       = v ? b : 0;
          cvv[li]      = v ? 1 : 0;
        }
      }
    }
    // 1c. slot and rank of every kept row (kNoRec: no row, key excluded, or
    //     sent to the global table)
    uint32_t rec[kTiledPer];
#pragma unroll
    for (int q = 0; q < kTiledPer; ++q) {
      rec[q] = kNoRec;
      if (!kept[q]) continue;
      int64_t s;
      if (key_is_empty<NW>(k[q])) {
        s = S;
        if (s_special == 0) s_special = 1;
      } else {
        s = find_or_insert<Shared, NW>(keys, S - 1, k[q], hash_key<NW>(k[q]), smem_probes);
      }
      if (s >= 0) {
        const uint32_t rank = atomicAdd(cnt + s, 1u);
        rec[q]              = (static_cast<uint32_t>(s) << 16) | rank;
      } else {
        const int64_t g = global_slot<NW>(t, k[q], max_probes);
        const int64_t r = t0 + threadIdx.x + q * kTiledBlock;
        if (g >= 0) {
          if constexpr (PART) accumulate_row_from<Global>(plan, psrc, G, g, r, t.status);
          else accumulate_row<Global>(plan, G, g, r, t.status);
        }
      }
    }
    __syncthreads();
    // 2. first position of each slot's rows; the rows listed in slot order
    {
      uint32_t c[kScanPer];
#pragma unroll
      for (int q = 0; q < kScanPer; ++q) {
        const uint32_t s = threadIdx.x * kScanPer + q;
        c[q]             = s <= S ? cnt[s] : 0u;
      }
      BlockScan(scan_tmp).ExclusiveSum(c, c);
#pragma unroll
      for (int q = 0; q < kScanPer; ++q) {
        const uint32_t s = threadIdx.x * kScanPer + q;
        if (s <= S) off[s] = c[q];
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kTiledPer; ++q)
      if (rec[q] != kNoRec)
        perm[off[rec[q] >> 16] + (rec[q] & 0xffffu)] = static_cast<uint16_t>(threadIdx.x + q * kTiledBlock);
    __syncthreads();
    // 3a. one thread per occupied slot: row count, and the VAR shift of each
    //     channel whose slot has none yet (the group's first valid non-NaN
    //     value in this tile), so that every chunk below folds against it
    uint32_t nchunk[kScanPer];
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) {
      const uint32_t s = threadIdx.x * kScanPer + q;
      const uint32_t c = s <= S ? cnt[s] : 0u;
      nchunk[q]        = (c + kChunk - 1) / kChunk;
      if (c == 0) continue;
      srows[s] += c;
      for (int ch = 0; ch < plan.nchan; ++ch) {
        const Channel& chan = plan.chan[ch];
        if (chan.a_k < 0) continue;
        uint64_t* kp = reinterpret_cast<uint64_t*>(smem + sl.acc_off[chan.a_k]) + s;
        if (*kp != kShiftUnset) continue;
        const uint64_t* cv = vals + static_cast<size_t>(ch) * tile_rows;
        const uint8_t* cvv = valid + static_cast<size_t>(ch) * tile_rows;
        for (uint32_t j = 0; j < c; ++j) {
          const uint32_t li = perm[off[s] + j];
          if (!cvv[li]) continue;
          const double xf = as_f64(cv[li], chan.ptype);
          if (xf != xf) continue;
          *kp = static_cast<uint64_t>(__double_as_longlong(xf));
          break;
        }
      }
    }
    // chunks of at most kChunk rows of one group: first chunk of each slot
    uint32_t total_chunks;
    BlockScan(scan_tmp).ExclusiveSum(nchunk, nchunk, total_chunks);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) {
      const uint32_t s = threadIdx.x * kScanPer + q;
      if (s > S) continue;
      const uint32_t n_s = (cnt[s] + kChunk - 1) / kChunk;
      for (uint32_t j = 0; j < n_s; ++j) cslot[nchunk[q] + j] = static_cast<uint16_t>(s);
      if (n_s > 0) coff[s] = nchunk[q];
    }
    __syncthreads();
    // 3b. every thread folds chunks in registers and merges each into its
    //     group's slot with shared atomics (a few chunks per group)
    const Level<Shared> L{base, &sl};
    for (uint32_t ci = threadIdx.x; ci < total_chunks; ci += blockDim.x) {
      const uint32_t s     = cslot[ci];
      const uint32_t j0    = (ci - coff[s]) * kChunk;
      const uint32_t first = off[s] + j0;
      const uint32_t len   = min(static_cast<uint32_t>(kChunk), cnt[s] - j0);
      for (int ch = 0; ch < plan.nchan; ++ch) {
        const Channel& chan = plan.chan[ch];
        const uint64_t* cv  = vals + static_cast<size_t>(ch) * tile_rows;
        const uint8_t* cvv  = valid + static_cast<size_t>(ch) * tile_rows;
        ChanAcc A;
        chan_acc_init(A);
        if (chan.a_k >= 0) A.k = reinterpret_cast<const uint64_t*>(smem + sl.acc_off[chan.a_k])[s];
#define GBX_FOLD_CHUNK(P) fold_chunk<P>(chan, cv, cvv, perm + first, len, A)
        switch (chan.ptype) {
          case P_I8: GBX_FOLD_CHUNK(P_I8); break;
          case P_I16: GBX_FOLD_CHUNK(P_I16); break;
          case P_I32: GBX_FOLD_CHUNK(P_I32); break;
          case P_I64: GBX_FOLD_CHUNK(P_I64); break;
          case P_U8: GBX_FOLD_CHUNK(P_U8); break;
          case P_U16: GBX_FOLD_CHUNK(P_U16); break;
          case P_U32: GBX_FOLD_CHUNK(P_U32); break;
          case P_U64: GBX_FOLD_CHUNK(P_U64); break;
          case P_F32: GBX_FOLD_CHUNK(P_F32); break;
          case P_F64: GBX_FOLD_CHUNK(P_F64); break;
          default: GBX_FOLD_CHUNK(P_BOOL); break;
        }
#undef GBX_FOLD_CHUNK
        merge_partial(chan, A, L, s, t.status);
      }
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) cnt[s] = 0;
    __syncthreads();
  }

  // merge the CTA's table into the global one
  for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) {
    uint64_t k[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = skeys[s * NW + w];
    const bool occupied = (s < S) ? !key_is_empty<NW>(k) : (s_special != 0);
    if (!occupied) continue;
    const int64_t g = global_slot<NW>(t, k, max_probes);
    if (g >= 0) merge_slot<Shared>(plan, Level<Shared>{base, &sl}, s, G, g, t.status);
  }
}

template <int NW, bool PART>
cudaError_t launch_tiled_nw(const Plan& p, const TableRef& t, const SmemLayout& sl, const TiledLayout& tl,
                            int64_t n, const PartBufs& pb, const uint32_t* n_part, int num_sms,
                            uint32_t smem_probes, uint32_t max_probes, cudaStream_t st)
{
  const void* fn = reinterpret_cast<const void*>(k_agg_tiled<NW, PART>);
  cudaError_t e  = ensure_dynamic_smem(fn, tl.total);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_agg_tiled<NW, PART>, kTiledBlock, tl.total)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int64_t ntiles = (n + tl.tile_rows - 1) / tl.tile_rows;
  const int grid       = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(num_sms) * per_sm)));
  k_agg_tiled<NW, PART><<<grid, kTiledBlock, tl.total, st>>>(p, t, sl, tl, n, pb, n_part, smem_probes, max_probes);
  return cudaGetLastError();
}

}  // namespace

bool tiled_fits(const SmemLayout& sl, int nchan)
{
  return sl.slots <= static_cast<uint32_t>(kTiledMaxSlots) && pick_tiled_layout(sl, nchan).tile_rows > 0;
}

cudaError_t launch_agg_tiled(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                             uint32_t smem_probes, uint32_t max_probes, cudaStream_t st)
{
  if (!tiled_fits(sl, p.nchan)) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  const TiledLayout tl = pick_tiled_layout(sl, p.nchan);
  const PartBufs none{};
  return p.key.nwords == 1 ? launch_tiled_nw<1, false>(p, t, sl, tl, n, none, nullptr, num_sms, smem_probes, max_probes, st)
                           : launch_tiled_nw<2, false>(p, t, sl, tl, n, none, nullptr, num_sms, smem_probes, max_probes, st);
}

cudaError_t launch_agg_tiled_part(const Plan& p, const TableRef& t, const SmemLayout& sl, const PartBufs& in,
                                  const uint32_t* n_rows, int64_t n, int num_sms, uint32_t smem_probes,
                                  uint32_t max_probes, cudaStream_t st)
{
  if (!tiled_fits(sl, p.nchan)) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  const TiledLayout tl = pick_tiled_layout(sl, p.nchan);
  return p.key.nwords == 1 ? launch_tiled_nw<1, true>(p, t, sl, tl, n, in, n_rows, num_sms, smem_probes, max_probes, st)
                           : launch_tiled_nw<2, true>(p, t, sl, tl, n, in, n_rows, num_sms, smem_probes, max_probes, st);
}

}  // namespace gbx
