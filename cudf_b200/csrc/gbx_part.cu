// gbx_part.cu -- radix-partitioned aggregation for high cardinality.
//
// When the groups do not fit per-warp tables, rows are first partitioned by
// the top bits of their key hash into P = 2^bits buckets of ~50-100 groups
// each (histogram, scans, scatter).  A warp then owns a bucket -- or, for a
// large bucket, a slice of it -- with a private shared-memory table
// (gbx_warpcore.cuh): no atomics on the row path.  A bucket handled by one
// warp has its rows ranked by group and each group folded in one lane's
// registers, then written straight into the output columns (dense rows
// reserved with one atomic per bucket); slices of a large bucket merge into a
// compact per-bucket region table that a last kernel writes out.  The reference keeps
// one global set of row indices sized by rows and updates N-row sparse columns
// with per-row atomics (hash/groupby.cu:424-504, 571-580); here every group's
// state lives in shared memory until it is final.

#include <algorithm>

#include "gbx_scan.hpp"
#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {
__device__ __forceinline__ uint32_t bucket_of(uint64_t h, int bits)
{
  return bits == 0 ? 0u : static_cast<uint32_t>(h >> (64 - bits));
}

__device__ __forceinline__ uint32_t lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Counter of bucket b for row r: with few buckets each bucket's counter is
// split into shards (by the row's 32-row batch, the same in the histogram and
// the scatter) so that warps do not all update the same address.
__device__ __forceinline__ uint32_t counter_of(uint32_t b, int64_t r, const PartPlan& pp)
{
  return (b << pp.shard_bits) | (static_cast<uint32_t>(r >> 5) & ((1u << pp.shard_bits) - 1u));
}

constexpr uint32_t kNoRank = 0xffffffffu;

// One whole bucket, rows [r0, r1), aggregated by one warp in four steps:
//   1. rank: each row finds or inserts its key in the warp's table (keys and
//      row counts only) and takes the next rank of its slot, lanes of a batch
//      in lane order, so that a group's rows keep their partitioned order;
//   2. scan: an exclusive scan of the slot counts gives each slot's first
//      position, and the occupied slots are listed with their counts;
//   3. permute: each row's values move to r0 + position + rank of `sorted`
//      (the same rows of a second set of copies), so that every group's rows
//      are contiguous;
//   4. emit: the bucket's groups get consecutive output rows; each group's
//      key columns and its run (first sorted row, row count) are written
//      there.
// The values are folded afterwards by k_part_fold, one thread per output
// row.  No accumulator lives in shared memory and no slot has more than one
// writer.  Keeping the generic accumulate/finalise code out of this kernel
// keeps its hot code within the instruction cache (a single kernel that also
// folded ran 2-2.5x slower from instruction-cache misses on B200).  The rank
// records live in the warp's shared memory (rec_smem, rec_rows entries) when
// the bucket fits, else in pp.rank_rec.
template <int NW>
__device__ __forceinline__ void part_bucket_ranked(const Plan& plan, const PartPlan& pp, const PartBufs& in,
                                                   const PartBufs& sorted, const WarpTable<NW>& T,
                                                   uint32_t* rec_smem, uint32_t rec_rows, const OutPlan& op,
                                                   int64_t r0, int64_t r1, uint32_t* scratch, int lane,
                                                   uint32_t* cta_nulls, int32_t* status)
{
  const PartSource src{&in};
  T.reset_keys(lane);
  uint32_t* cnt      = T.rows();
  const uint32_t len = static_cast<uint32_t>(r1 - r0);
  uint32_t* rec      = len <= rec_rows ? rec_smem : pp.rank_rec + r0;

  // 1. rank
  int64_t r = r0 + lane;
  uint64_t k[NW];
  bool act = r < r1 && src.key<NW>(r, k);
  for (int64_t base = r0; base < r1; base += 32) {
    const int64_t rn = base + 32 + lane;
    uint64_t kn[NW];
    const bool actn = rn < r1 && src.key<NW>(rn, kn);
    uint32_t slot;
    const int state = warp_find_or_insert<NW>(T, plan.acc, act, k, lane, slot);
    if (state == ST_SPILL) atomicOr(status, S_TABLE_FULL);  // bucket larger than its table: host retries
    const bool found      = state == ST_FOUND;
    const uint32_t fm     = __ballot_sync(kFull, found);
    const uint32_t peers  = found ? __match_any_sync(fm, slot) : 0u;
    const uint32_t before = __popc(peers & lanemask_lt(lane));
    const uint32_t rank   = found ? cnt[slot] + before : 0u;
    __syncwarp();
    if (found && before == 0) cnt[slot] += __popc(peers);
    if (act) rec[r - r0] = found ? ((slot << 16) | rank) : kNoRank;
    __syncwarp();
    r   = rn;
    act = actn;
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = kn[w];
  }

  // 2. scan: slot counts -> first positions (in place); occupied slots with
  // their counts (count << 16 | slot) into scratch
  uint32_t run = 0, ngroups = 0;
  for (uint32_t s0 = 0; s0 <= T.S; s0 += 32) {
    const uint32_t s = s0 + lane;
    const uint32_t c = s <= T.S ? cnt[s] : 0u;
    uint32_t incl    = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += y;
    }
    if (s <= T.S) cnt[s] = run + incl - c;
    const uint32_t bal = __ballot_sync(kFull, c > 0);
    if (c > 0) scratch[ngroups + __popc(bal & lanemask_lt(lane))] = (c << 16) | s;
    run += __shfl_sync(kFull, incl, 31);
    ngroups += __popc(bal);
  }
  __syncwarp();

  // 3. permute
  for (uint32_t i = lane; i < len; i += 32) {
    const uint32_t v = rec[i];
    if (v == kNoRank) continue;
    const int64_t from = r0 + i;
    const int64_t to   = r0 + cnt[v >> 16] + (v & 0xffffu);
    for (int c = 0; c < plan.nchan; ++c) {
      const PartCol& a = in.col[c];
      const PartCol& b = sorted.col[c];
      store_bits(const_cast<void*>(b.vals), to, a.width, load_bits(a.vals, from, a.width));
      if (a.valid != nullptr) const_cast<uint8_t*>(b.valid)[to] = __ldg(a.valid + from);
    }
  }
  __syncwarp();  // orders the warp's stores before its loads below
  if (ngroups == 0) return;

  // 4. emit: output rows reserved with one atomic; each group's key columns
  // and (first sorted row, row count) at its output row
  unsigned long long ob = 0;
  if (lane == 0) ob = atomicAdd(pp.out_counter, static_cast<unsigned long long>(ngroups));
  ob                   = __shfl_sync(kFull, ob, 0);
  const uint64_t* keys = T.keys();
  const NullSink sink{op.null_counts, cta_nulls};
  for (uint32_t g0 = 0; g0 < ngroups; g0 += 32) {
    const int64_t base = static_cast<int64_t>(ob + g0);
    const bool active  = g0 + lane < ngroups;
    const uint32_t ent = active ? scratch[g0 + lane] : 0u;
    const uint32_t ss  = ent & 0xffffu;
    const uint32_t act = __ballot_sync(kFull, active);
    uint64_t k2[2]     = {0, 0};
    if (active) {
#pragma unroll
      for (int w = 0; w < NW; ++w) k2[w] = keys[ss * NW + w];
      if (ss == T.S) k2[0] = k2[1] = kEmptyWord;
      pp.group_run[base + lane] = make_uint2(static_cast<uint32_t>(r0) + cnt[ss], ent >> 16);
    }
    warp_write_keys(plan, op, active, k2, base, lane, act, sink);
  }
}

// Channel c's outputs for a warp's 32 output rows [base, base + 32): lane i
// folds its group's run of sorted rows into registers (ChanAcc) and writes
// the channel's outputs.  Specialised on the channel's physical type PT, so
// the accumulate and finalise code has no type switches left.  Warps own
// aligned 32-row runs of output rows, so validity words are stored whole.
template <int PT>
__device__ __forceinline__ void fold_channel(const Plan& plan, const OutPlan& op, const PartCol& pc, int c,
                                             uint2 run, bool active, int64_t base, int lane, uint32_t act,
                                             uint32_t* cta_nulls)
{
  using Word        = typename std::conditional<pt_width(PT) == 1, uint8_t,
                        typename std::conditional<pt_width(PT) == 2, uint16_t,
                          typename std::conditional<pt_width(PT) == 4, uint32_t,
                                                    unsigned long long>::type>::type>::type;
  const Channel& ch     = plan.chan[c];
  const uint32_t roles  = chan_roles(ch);
  const Word* vals      = reinterpret_cast<const Word*>(pc.vals);
  ChanAcc A;
  chan_acc_init(A);
  // the run's first kFoldBatch rows are loaded together (one round trip for
  // almost every group at high cardinality), then folded in row order
  constexpr uint32_t kFoldBatch = 4;
  uint64_t pre[kFoldBatch];
  bool pok[kFoldBatch];
#pragma unroll
  for (uint32_t j = 0; j < kFoldBatch; ++j) {
    const int64_t r = static_cast<int64_t>(run.x) + j;
    const bool in   = j < run.y;
    pre[j]          = in ? static_cast<uint64_t>(__ldg(vals + r)) : 0;
    pok[j]          = in && (pc.valid == nullptr || __ldg(pc.valid + r) != 0);
  }
#pragma unroll
  for (uint32_t j = 0; j < kFoldBatch; ++j)
    if (pok[j]) chan_acc_add<PT>(ch, roles, A, pre[j]);
  for (uint32_t j = kFoldBatch; j < run.y; ++j) {
    const int64_t r = static_cast<int64_t>(run.x) + j;
    const uint64_t b = __ldg(vals + r);
    if (pc.valid == nullptr || __ldg(pc.valid + r) != 0) chan_acc_add<PT>(ch, roles, A, b);
  }
  const RegView V{A, run.y};
  const int64_t g = base + lane;
  // Shared by the channel's outputs, once per group: the mean (one FP64
  // division) and, with VAR/STD, the centred sum of squares
  // M2 = sum (x-K)^2 - S1 (S1 / n), S1 = sum (x - K) (shifted_sum: the
  // folded shifted sum of a floating channel, the exact integer difference
  // otherwise).  MEAN divides the signed INT64 SUM of an integer column.
  const bool is_float = PT == P_F32 || PT == P_F64;
  const double n      = static_cast<double>(A.cnt);
  const double sum_m  = is_float ? __longlong_as_double(static_cast<long long>(A.sum))
                                 : static_cast<double>(static_cast<int64_t>(A.sum));
  const double mean   = (roles & R_SUM) && A.cnt > 0 ? sum_m / n : 0.0;
  double m2           = 0.0;
  if ((roles & R_VAR) && A.cnt > 0) {
    if (A.k == kShiftUnset) {
      m2 = A.s2;  // NaN inputs only
    } else {
      const double K  = __longlong_as_double(static_cast<long long>(A.k));
      const double S1 = shifted_sum(is_float, PT, A.sum, static_cast<uint64_t>(__double_as_longlong(A.s1)), A.cnt, K);
      m2              = A.s2 - S1 * (S1 / n);
      if (m2 < 0.0) m2 = 0.0;
    }
  }
  for (int o = 0; o < op.nout; ++o) {
    const OutCol& oc = op.out[o];
    if (oc.chan != c) continue;
    bool valid = false;
    uint64_t v = 0;
    if (active) {
      if (oc.kind == GBX_AGG_MEAN && oc.out_ptype == P_F64) {
        valid = A.cnt > 0;
        v     = valid ? static_cast<uint64_t>(__double_as_longlong(mean)) : 0;
      } else if (oc.kind == GBX_AGG_VARIANCE || oc.kind == GBX_AGG_STD || oc.kind == GBX_AGG_M2) {
        // M2 (group_m2.cu): the centred sum of squares itself, null without values
        const int64_t nn   = A.cnt;
        const int64_t ddof = oc.kind == GBX_AGG_M2 ? 0 : oc.ddof;
        valid              = nn > 0 && nn - ddof > 0;
        if (valid) {
          double var = A.k == kShiftUnset || oc.kind == GBX_AGG_M2 ? m2 : m2 / static_cast<double>(nn - ddof);
          if (oc.kind == GBX_AGG_STD) var = sqrt(var);
          v = static_cast<uint64_t>(__double_as_longlong(var));
        }
      } else {
        v = finalize_from<PT>(ch, oc, V, valid);
      }
    }
    if (active) store_bits(oc.data, g, oc.out_width, v);
    if (oc.mask != nullptr) {
      const uint32_t bits = __ballot_sync(kFull, active && valid);
      if (lane == 0) {
        oc.mask[base >> 5] = bits;
        const uint32_t nulls = __popc(act & ~bits);
        if (nulls != 0) atomicAdd(cta_nulls + kMaxKeyCols + o, nulls);
      }
    }
  }
}

}  // namespace

// Rows per bucket (warp-aggregated: one atomic per bucket present in a warp).
template <int NW>
__global__ void k_part_hist(const __grid_constant__ KeyPlan kp, int64_t n, const __grid_constant__ PartPlan pp)
{
  const int lane       = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31); base < n;
       base += stride) {
    const int64_t r = base + lane;
    uint64_t k[NW];
    const bool act    = r < n && pack_key<NW>(kp, r, k);
    const uint32_t b  = act ? bucket_of(hash_key<NW>(k), pp.bits) : 0xffffffffu;
    const uint32_t pe = __match_any_sync(kFull, b);
    if (act && (__ffs(pe) - 1) == lane) atomicAdd(pp.counts + counter_of(b, r, pp), static_cast<uint32_t>(__popc(pe)));
  }
}

__global__ void k_part_slices(const __grid_constant__ PartPlan pp)
{
  const uint32_t P = 1u << pp.bits;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= P; b += gridDim.x * blockDim.x) {
    if (b == P) {
      pp.nslices[b] = 0;
      pp.multi[b]   = 0;
    } else {
      // a bucket of at most slice_rows rows is a whole-bucket item of
      // k_part_ranked, not a slice
      const uint32_t o0 = pp.offsets[b << pp.shard_bits];
      const uint32_t o1 = pp.offsets[(b + 1) << pp.shard_bits];
      if (o1 < o0) atomicOr(pp.status, S_CHECK_FAILED);  // rows not in bucket order
      const uint32_t c  = o1 >= o0 ? o1 - o0 : 0u;
      const uint32_t ns = (c + pp.slice_rows - 1) / pp.slice_rows;
      pp.nslices[b]     = ns > 1 ? ns : 0u;
      pp.multi[b]       = ns > 1 ? 1u : 0u;
    }
  }
}

// Bucket of every work item (one thread per bucket writes its slices).
__global__ void k_part_items(const __grid_constant__ PartPlan pp)
{
  const uint32_t P = 1u << pp.bits;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < P; b += gridDim.x * blockDim.x) {
    const uint32_t i0 = pp.item_start[b];
    const uint32_t ns = pp.nslices[b];
    for (uint32_t j = 0; j < ns; ++j) pp.item_bucket[i0 + j] = b;
  }
}

// Writes each row's packed key, resolved values and validity to its bucket.
// Each warp takes 4 batches of 32 rows at a time so that the 4 batches'
// cursor atomics (whose results the writes need) are in flight together.
template <int NW>
__global__ void k_part_scatter(const __grid_constant__ Plan plan, int64_t n, const __grid_constant__ PartPlan pp,
                               const __grid_constant__ PartBufs out)
{
  constexpr int U         = 4;
  const int lane          = threadIdx.x & 31;
  const int64_t warp      = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps    = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const RowSource src{&plan};
  for (int64_t base = warp * 32 * U; base < n; base += nwarps * 32 * U) {
    uint64_t k[U][NW];
    bool act[U];
    uint32_t pe[U], pos[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t r  = base + u * 32 + lane;
      act[u]           = r < n && src.key<NW>(r, k[u]);
      const uint32_t b = act[u] ? bucket_of(hash_key<NW>(k[u]), pp.bits) : 0xffffffffu;
      pe[u]            = __match_any_sync(kFull, b);
      pos[u]           = 0;
      if (act[u] && lane == __ffs(pe[u]) - 1)
        pos[u] = atomicAdd(pp.cursor + counter_of(b, base + u * 32 + lane, pp), static_cast<uint32_t>(__popc(pe[u])));
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t p0 = __shfl_sync(kFull, pos[u], __ffs(pe[u]) - 1);
      if (!act[u]) continue;
      const int64_t r   = base + u * 32 + lane;
      const uint32_t at = p0 + __popc(pe[u] & lanemask_lt(lane));
#pragma unroll
      for (int w = 0; w < NW; ++w) const_cast<uint64_t*>(out.keys[w])[at] = k[u][w];
      for (int c = 0; c < plan.nchan; ++c) {
        uint64_t bits = 0;
        const bool v  = src.value(c, r, bits, pp.status);
        store_bits(const_cast<void*>(out.col[c].vals), at, out.col[c].width, v ? bits : 0);
        if (out.col[c].valid != nullptr) const_cast<uint8_t*>(out.col[c].valid)[at] = v ? 1 : 0;
      }
    }
  }
}

// Per-warp shared memory of k_part_ranked: a keys-and-counts table
// (sl.slots + 1 slots), the occupied-slot list and the rank records.
struct RankedLayout {
  uint32_t stride;       // bytes per warp
  uint32_t scratch_off;  // sl.slots + 32 u32
  uint32_t rec_off;      // rec_rows u32
  uint32_t rec_rows;
};

// Whole buckets, claimed a few at a time, each through part_bucket_ranked.
// `sl` describes the table part of each warp's shared memory (keys_off,
// rows_off); it has no accumulator arrays.
constexpr int kRankedCtasPerSm = 4;

template <int NW>
__global__ void __launch_bounds__(256, kRankedCtasPerSm) k_part_ranked(const __grid_constant__ Plan plan,
                                                       const __grid_constant__ PartPlan pp,
                                                       const __grid_constant__ PartBufs in,
                                                       const __grid_constant__ PartBufs sorted,
                                                       const __grid_constant__ SmemLayout sl,
                                                       const __grid_constant__ RankedLayout rl,
                                                       const __grid_constant__ OutPlan op)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane         = threadIdx.x & 31;
  unsigned char* wmem    = smem + static_cast<size_t>(threadIdx.x >> 5) * rl.stride;
  const WarpTable<NW> T{wmem, &sl, sl.slots};
  uint32_t* scratch      = reinterpret_cast<uint32_t*>(wmem + rl.scratch_off);
  uint32_t* rec          = reinterpret_cast<uint32_t*>(wmem + rl.rec_off);
  const uint32_t P       = 1u << pp.bits;
  __shared__ uint32_t s_nulls[kNullSlots];
  cta_nulls_zero(s_nulls);

  constexpr int kClaim = 4;  // buckets claimed per atomic
  unsigned long long claimed = 0, claim_end = 0;
  for (;;) {
    if (claimed == claim_end) {
      unsigned long long c0 = 0;
      if (lane == 0) c0 = atomicAdd(pp.bucket_counter, static_cast<unsigned long long>(kClaim));
      claimed   = __shfl_sync(kFull, c0, 0);
      claim_end = claimed + kClaim;
    }
    const unsigned long long b = claimed++;
    if (b >= P) break;
    if (pp.multi[b] != 0) continue;  // sliced: k_part_agg
    const int64_t r0 = pp.offsets[b << pp.shard_bits];
    const int64_t r1 = pp.offsets[(b + 1) << pp.shard_bits];
    if (r1 == r0) continue;
    part_bucket_ranked<NW>(plan, pp, in, sorted, T, rec, rl.rec_rows, op, r0, r1, scratch, lane, s_nulls,
                           pp.status);
    __syncwarp();
  }
  cta_nulls_flush(s_nulls, op.null_counts);
}

// Shared memory of k_part_ranked_cta: a keys table of slots + 1 entries
// (slot `slots` is the reserved all-ones key), slots + 2 counters (rows of
// each slot, then each slot's first position, then the total), the occupied
// slots in slot order and rec_rows rank records.
struct CtaRankLayout {
  uint32_t slots;  // power of two, a multiple of the block size
  uint32_t cnt_off;
  uint32_t list_off;
  uint32_t rec_off;
  uint32_t rec_rows;
  uint32_t total;
};

constexpr int kCtaRankThreads = 256;
constexpr int kCtaBatch       = 4;  // rows a thread loads together in k_part_ranked_cta's row loops
// Rank records of k_part_ranked_cta: slot (up to 4,096, 13 bits) above a
// 19-bit rank, so that one CTA takes buckets of up to 2^19 rows.
constexpr int kCtaRankBits          = 19;
constexpr uint32_t kCtaRankMask     = (1u << kCtaRankBits) - 1u;
constexpr uint32_t kCtaMaxSliceRows = 1u << kCtaRankBits;

// Exclusive scan of one 64-bit value per thread over the block; *total gets
// the block's sum.  `part` holds one entry per warp.  Ends with the block
// synchronised.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* part, uint64_t* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint64_t incl  = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, incl, d);
    if (lane >= d) incl += y;
  }
  if (lane == 31) part[warp] = incl;
  __syncthreads();
  uint64_t before = 0, all = 0;
  for (int w = 0; w < nwarps; ++w) {
    const uint64_t p = part[w];
    before += w < warp ? p : 0;
    all += p;
  }
  *total = all;
  __syncthreads();  // `part` may be reused after the return
  return before + incl - v;
}

// Whole buckets, one per CTA at a time: the same four steps as
// part_bucket_ranked with the bucket's rows spread over the block and one
// table of cl.slots slots for the whole CTA, so that a bucket may hold a few
// thousand groups (2^8 times fewer buckets than the warp form needs for the
// same groups: one radix pass less).  Each row's rank within its slot comes
// from a 32-bit shared atomic, so a group's rows are contiguous in `sorted`
// but not in partitioned order (floating-point sums may round differently
// from run to run; every other result is order-independent).
template <int NW>
__global__ void __launch_bounds__(kCtaRankThreads, 4) k_part_ranked_cta(const __grid_constant__ Plan plan,
                                                                      const __grid_constant__ PartPlan pp,
                                                                      const __grid_constant__ PartBufs in,
                                                                      const __grid_constant__ PartBufs sorted,
                                                                      const __grid_constant__ CtaRankLayout cl,
                                                                      const __grid_constant__ OutPlan op)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t s_nulls[kNullSlots];
  __shared__ uint64_t s_part[kCtaRankThreads / 32];
  __shared__ unsigned long long s_claim, s_out;
  const uint32_t S       = cl.slots;
  uint64_t* keys         = reinterpret_cast<uint64_t*>(smem);
  const uint32_t keys_sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  uint32_t* cnt          = reinterpret_cast<uint32_t*>(smem + cl.cnt_off);
  uint32_t* list         = reinterpret_cast<uint32_t*>(smem + cl.list_off);
  uint32_t* rec_smem     = reinterpret_cast<uint32_t*>(smem + cl.rec_off);
  const PartSource src{&in};
  const uint32_t P   = 1u << pp.bits;
  const int lane     = threadIdx.x & 31;
  const uint32_t tid = threadIdx.x;
  const NullSink sink{op.null_counts, s_nulls};
  cta_nulls_zero(s_nulls);

  for (;;) {
    if (tid == 0) s_claim = atomicAdd(pp.bucket_counter, 1ull);
    __syncthreads();
    const unsigned long long b = s_claim;
    __syncthreads();  // every thread has read s_claim before thread 0 claims again
    if (b >= P) break;
    if (pp.multi[b] != 0) continue;  // sliced: k_part_agg
    const int64_t r0 = pp.offsets[b << pp.shard_bits];
    const int64_t r1 = pp.offsets[(b + 1) << pp.shard_bits];
    if (r1 == r0) continue;
    const uint32_t len = static_cast<uint32_t>(r1 - r0);
    uint32_t* rec      = len <= cl.rec_rows ? rec_smem : pp.rank_rec + r0;

    for (uint32_t s = tid; s <= S + 1; s += blockDim.x) {
      if (s <= S) {
#pragma unroll
        for (int w = 0; w < NW; ++w) keys[s * NW + w] = kEmptyWord;
      }
      cnt[s] = 0;
    }
    __syncthreads();

    // 1. rank (kCtaBatch rows a thread: their key loads in flight together)
    for (uint32_t i0 = tid; i0 < len; i0 += kCtaBatch * blockDim.x) {
      uint64_t k[kCtaBatch][NW];
      bool act[kCtaBatch];
#pragma unroll
      for (int q = 0; q < kCtaBatch; ++q) {
        const uint32_t i = i0 + q * blockDim.x;
        act[q]           = i < len && src.key<NW>(r0 + i, k[q]);
      }
#pragma unroll
      for (int q = 0; q < kCtaBatch; ++q) {
        const uint32_t i = i0 + q * blockDim.x;
        if (i >= len) break;
        uint32_t v = kNoRank;
        if (act[q]) {
          int64_t slot = S;
          if (!key_is_empty<NW>(k[q])) {
            slot = find_or_insert<Shared, NW>(keys_sa, S - 1, k[q], hash_key<NW>(k[q]), S);
            if (slot < 0) atomicOr(pp.status, S_TABLE_FULL);  // more groups than the table: host retries
          }
          if (slot >= 0) {
            const uint32_t rank = atomicAdd(cnt + slot, 1u);
            v                   = (static_cast<uint32_t>(slot) << kCtaRankBits) | rank;
          }
        }
        rec[i] = v;
      }
    }
    __syncthreads();

    // 2. scan: first position of every slot (in place), occupied slots listed
    // in slot order; each thread scans S / blockDim.x consecutive slots
    const uint32_t per = S / blockDim.x;
    const uint32_t sb  = tid * per;
    uint32_t csum = 0, occ = 0;
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t c = cnt[sb + j];
      csum += c;
      occ += c != 0;
    }
    uint64_t total;
    const uint64_t ex = block_exclusive_scan((static_cast<uint64_t>(occ) << 32) | csum, s_part, &total);
    uint32_t pos = static_cast<uint32_t>(ex), gi = static_cast<uint32_t>(ex >> 32);
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t c = cnt[sb + j];
      cnt[sb + j]      = pos;
      pos += c;
      if (c != 0) list[gi++] = sb + j;
    }
    const uint32_t tot_rows = static_cast<uint32_t>(total), tot_groups = static_cast<uint32_t>(total >> 32);
    const uint32_t cs       = cnt[S];  // the reserved slot's rows (read by all before thread 0 rewrites it)
    const uint32_t ngroups  = tot_groups + (cs != 0);
    __syncthreads();
    if (tid == 0) {
      cnt[S]     = tot_rows;
      cnt[S + 1] = tot_rows + cs;
      if (cs != 0) list[tot_groups] = S;
      s_out = atomicAdd(pp.out_counter, static_cast<unsigned long long>(ngroups));
    }
    __syncthreads();

    // 3. permute (kCtaBatch rows a thread, each channel's loads in flight
    // together before its stores)
    for (uint32_t i0 = tid; i0 < len; i0 += kCtaBatch * blockDim.x) {
      int64_t to[kCtaBatch];
#pragma unroll
      for (int q = 0; q < kCtaBatch; ++q) {
        const uint32_t i = i0 + q * blockDim.x;
        const uint32_t v = i < len ? rec[i] : kNoRank;
        to[q]            = v == kNoRank ? -1 : r0 + cnt[v >> kCtaRankBits] + (v & kCtaRankMask);
      }
      for (int c = 0; c < plan.nchan; ++c) {
        const PartCol& a = in.col[c];
        const PartCol& d = sorted.col[c];
        uint64_t x[kCtaBatch];
        uint8_t ok[kCtaBatch];
#pragma unroll
        for (int q = 0; q < kCtaBatch; ++q) {
          const int64_t from = r0 + i0 + q * blockDim.x;
          x[q]               = to[q] >= 0 ? load_bits(a.vals, from, a.width) : 0;
          ok[q]              = to[q] >= 0 && a.valid != nullptr ? __ldg(a.valid + from) : 0;
        }
#pragma unroll
        for (int q = 0; q < kCtaBatch; ++q) {
          if (to[q] < 0) continue;
          store_bits(const_cast<void*>(d.vals), to[q], a.width, x[q]);
          if (a.valid != nullptr) const_cast<uint8_t*>(d.valid)[to[q]] = ok[q];
        }
      }
    }

    // 4. emit: the bucket's groups at output rows s_out + [0, ngroups), each
    // with its key columns and (first sorted row, row count)
    const unsigned long long ob = s_out;
    for (uint32_t g0 = tid & ~31u; g0 < ngroups; g0 += blockDim.x) {
      const bool active = g0 + lane < ngroups;
      const uint32_t ss = active ? list[g0 + lane] : 0u;
      const uint32_t act = __ballot_sync(kFull, active);
      uint64_t k2[2]     = {0, 0};
      const int64_t base = static_cast<int64_t>(ob + g0);
      if (active) {
#pragma unroll
        for (int w = 0; w < NW; ++w) k2[w] = keys[ss * NW + w];
        if (ss == S) k2[0] = k2[1] = kEmptyWord;
        pp.group_run[base + lane] = make_uint2(static_cast<uint32_t>(r0) + cnt[ss], cnt[ss + 1] - cnt[ss]);
      }
      warp_write_keys(plan, op, active, k2, base, lane, act, sink);
    }
    __syncthreads();  // the table is reset for the next bucket
  }
  cta_nulls_flush(s_nulls, op.null_counts);
}

// Channel c's value outputs of the groups k_part_ranked emitted (output rows
// [0, *pp.out_counter): it runs right after k_part_ranked, before any slice
// adds output rows), one thread per group; one launch per channel, each
// specialised on that channel's physical type PT.
template <int PT>
__global__ void __launch_bounds__(256) k_part_fold(const __grid_constant__ Plan plan,
                                                   const __grid_constant__ PartPlan pp,
                                                   const __grid_constant__ PartBufs sorted,
                                                   const __grid_constant__ OutPlan op, int c)
{
  __shared__ uint32_t s_nulls[kNullSlots];
  cta_nulls_zero(s_nulls);
  const int64_t G       = static_cast<int64_t>(*pp.out_counter);
  const int lane        = threadIdx.x & 31;
  const int64_t wstride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31);
  // each group's (first row, rows) is loaded one iteration ahead
  uint2 next = base + lane < G ? pp.group_run[base + lane] : make_uint2(0u, 0u);
  for (; base < G; base += wstride) {
    const bool active  = base + lane < G;
    const uint2 run    = next;
    const int64_t nb   = base + wstride + lane;
    next               = nb < G ? pp.group_run[nb] : make_uint2(0u, 0u);
    const uint32_t act = __ballot_sync(kFull, active);
    fold_channel<PT>(plan, op, sorted.col[c], c, run, active, base, lane, act, s_nulls);
  }
  cta_nulls_flush(s_nulls, op.null_counts);
}

template <int PT>
cudaError_t launch_fold(const Plan& p, const PartPlan& pp, const PartBufs& sorted, const OutPlan& op, int c,
                        int num_sms, cudaStream_t st)
{
  int per_sm    = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_part_fold<PT>, 256, 0);
  if (e != cudaSuccess) return e;
  k_part_fold<PT><<<num_sms * std::max(per_sm, 1), 256, 0, st>>>(p, pp, sorted, op, c);
  return cudaGetLastError();
}

// Slices of the buckets larger than slice_rows (see the file comment):
// blockDim.x / 32 warp tables of sl.total bytes with accumulators, merged
// into the bucket's region table.
template <int NW, int NCH>
__global__ void __launch_bounds__(256, 2) k_part_agg(const __grid_constant__ Plan plan, const __grid_constant__ PartPlan pp, const __grid_constant__ PartBufs in, const __grid_constant__ TableRef t, const __grid_constant__ SmemLayout sl)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane   = threadIdx.x & 31;
  const int warp   = threadIdx.x >> 5;
  WarpTable<NW> T{smem + static_cast<size_t>(warp) * sl.total, &sl, sl.slots};
  const PartSource src{&in};
  const uint32_t P          = 1u << pp.bits;
  const uint64_t items      = pp.item_start[P];
  const Level<Global> Gl    = global_level(t);
  const uint64_t* keys      = T.keys();

  constexpr int kClaim = 4;  // work items claimed per atomic
  unsigned long long claimed = 0, claim_end = 0;
  for (;;) {
    if (claimed == claim_end) {
      unsigned long long c0 = 0;
      if (lane == 0) c0 = atomicAdd(pp.item_counter, static_cast<unsigned long long>(kClaim));
      claimed   = __shfl_sync(kFull, c0, 0);
      claim_end = claimed + kClaim;
    }
    const unsigned long long item = claimed++;
    if (item >= items) break;
    const uint32_t b   = pp.item_bucket[item];
    const uint32_t ns  = pp.nslices[b];
    const uint64_t j   = item - pp.item_start[b];
    const uint64_t b0  = pp.offsets[b << pp.shard_bits];
    const uint64_t b1  = pp.offsets[(b + 1) << pp.shard_bits];
    const uint64_t len = b1 >= b0 ? b1 - b0 : 0;
    const int64_t r0   = static_cast<int64_t>(b0 + len * j / ns);
    const int64_t r1   = static_cast<int64_t>(b0 + len * (j + 1) / ns);

    T.reset(plan.acc, lane);
    bool special = false;
    int64_t r = r0 + lane;
    uint64_t k[NW];
    bool act  = r < r1 && src.key<NW>(r, k);
    RowVals<NCH> v;
    load_row_values(plan, src, act, r, v, t.status);
    for (int64_t base = r0; base < r1; base += 32) {
      const int64_t rn = base + 32 + lane;
      uint64_t kn[NW];
      const bool actn = rn < r1 && src.key<NW>(rn, kn);
      RowVals<NCH> vn;
      load_row_values(plan, src, actn, rn, vn, t.status);

      uint32_t slot;
      const int state = warp_find_or_insert<NW>(T, plan.acc, act, k, lane, slot);
      if (__any_sync(kFull, state == ST_FOUND && slot == T.S)) special = true;
      if (state == ST_SPILL) atomicOr(t.status, S_TABLE_FULL);  // bucket larger than its table: host retries
      warp_accumulate(plan, T.tb, sl, state == ST_FOUND, slot, v, lane);

      r   = rn;
      act = actn;
#pragma unroll
      for (int w = 0; w < NW; ++w) k[w] = kn[w];
      v = vn;
    }

    {
      const Level<Shared> L{static_cast<uint32_t>(__cvta_generic_to_shared(T.tb)), &sl};
      const uint64_t rbase = static_cast<uint64_t>(pp.region[b]) * pp.region_slots;
      for (uint32_t s = lane; s <= T.S; s += 32) {
        uint64_t kw[NW];
#pragma unroll
        for (int w = 0; w < NW; ++w) kw[w] = keys[s * NW + w];
        const bool occ = (s < T.S) ? !key_is_empty<NW>(kw) : special;
        if (!occ) continue;
        int64_t g;
        if (s == T.S) {
          g = global_slot<NW>(t, kw, 1);
        } else {
          g = find_or_insert<Global, NW>(reinterpret_cast<uint64_t>(t.keys + rbase * NW), pp.region_slots - 1, kw,
                                         hash_key<NW>(kw), pp.region_slots);
          if (g < 0) atomicOr(t.status, S_TABLE_FULL);
          else g += static_cast<int64_t>(rbase);
        }
        if (g >= 0) merge_slot<Shared>(plan, L, s, Gl, g, t.status);
      }
    }
    __syncwarp();
  }
}

// Writes out the groups of the region tables (and the reserved all-ones slot).
template <int NW>
__global__ void k_part_region_finalize(const __grid_constant__ Plan plan, const __grid_constant__ PartPlan pp, const __grid_constant__ TableRef t, const __grid_constant__ OutPlan op)
{
  __shared__ uint32_t scratch_all[8][32];
  __shared__ uint32_t s_nulls[kNullSlots];
  cta_nulls_zero(s_nulls);
  const int lane         = threadIdx.x & 31;
  uint32_t* scratch      = scratch_all[(threadIdx.x >> 5) & 7];
  const uint64_t nslots  = t.cap + 1;
  const uint64_t stride  = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const GlobalAccs A{&t};
  for (uint64_t s0 = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~uint64_t(31); s0 < nslots;
       s0 += stride) {
    const uint64_t s = s0 + lane;
    bool occ         = false;
    if (s < t.cap) {
      uint64_t kw[NW];
#pragma unroll
      for (int w = 0; w < NW; ++w) kw[w] = t.keys[s * NW + w];
      occ = !key_is_empty<NW>(kw);
    } else if (s == t.cap) {
      occ = *t.special_used != 0;
    }
    const uint32_t bal = __ballot_sync(kFull, occ);
    if (bal == 0) continue;
    const int cnt = __popc(bal);
    if (occ) scratch[__popc(bal & lanemask_lt(lane))] = static_cast<uint32_t>(s - s0);
    __syncwarp();
    unsigned long long ob = 0;
    if (lane == 0) ob = atomicAdd(pp.out_counter, static_cast<unsigned long long>(cnt));
    ob                = __shfl_sync(kFull, ob, 0);
    const bool active = lane < cnt;
    const uint64_t ss = active ? s0 + scratch[lane] : 0;
    uint64_t k2[2]    = {0, 0};
    if (active) {
      if (ss == t.cap) {
        k2[0] = k2[1] = kEmptyWord;
      } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) k2[w] = t.keys[ss * NW + w];
      }
    }
    warp_write_groups(plan, op, A, active, ss, k2, static_cast<int64_t>(ob), lane, s_nulls);
    __syncwarp();
  }
  cta_nulls_flush(s_nulls, op.null_counts);
}

// ---------------------------------------------------------------- launchers

namespace {
inline int grid_rows(int64_t n, int block, int max_blocks)
{
  int64_t b = (n + block - 1) / block;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, max_blocks)));
}
}  // namespace

cudaError_t launch_part_hist(const KeyPlan& kp, int64_t n, const PartPlan& pp, int num_sms, cudaStream_t st)
{
  const size_t counters = (size_t(1) << (pp.bits + pp.shard_bits)) + 1;
  cudaError_t e         = cudaMemsetAsync(pp.counts, 0, counters * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  const int grid = grid_rows(n, 256, num_sms * 8);
  if (kp.nwords == 1) k_part_hist<1><<<grid, 256, 0, st>>>(kp, n, pp);
  else k_part_hist<2><<<grid, 256, 0, st>>>(kp, n, pp);
  return cudaGetLastError();
}

cudaError_t launch_part_layout(const PartPlan& pp, void* temp, size_t* temp_bytes, int num_sms, cudaStream_t st,
                               bool offsets_ready)
{
  const int items    = (1 << pp.bits) + 1;
  const int counters = (1 << (pp.bits + pp.shard_bits)) + 1;
  if (temp == nullptr) {  // sized for the largest scan (counters >= items)
    return scan_exclusive_u32(nullptr, nullptr, counters, nullptr, temp_bytes, st);
  }
  cudaError_t e;
  if (!offsets_ready) {
    e = scan_exclusive_u32(pp.counts, pp.offsets, counters, temp, temp_bytes, st);
    if (e != cudaSuccess) return e;
  }
  k_part_slices<<<grid_rows(items, 256, num_sms * 4), 256, 0, st>>>(pp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan_exclusive_u32(pp.nslices, pp.item_start, items, temp, temp_bytes, st)) != cudaSuccess) return e;
  if ((e = scan_exclusive_u32(pp.multi, pp.region, items, temp, temp_bytes, st)) != cudaSuccess) return e;
  if (offsets_ready) return cudaSuccess;  // cursors are only used by the one-pass scatter
  return cudaMemcpyAsync(pp.cursor, pp.offsets, (counters - 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
}

namespace {
// offsets[b] = i for the buckets b in (bucket of row i - 1, bucket of row i]
// (row -1 in bucket -1, row *n_rows in bucket P): every bucket's first row,
// each entry written once.
template <int NW>
__global__ void k_part_bounds(const uint64_t* k0, const uint64_t* k1, const uint32_t* n_rows, int bits,
                              uint32_t* offsets)
{
  const int64_t n      = static_cast<int64_t>(*n_rows);
  const int64_t P      = int64_t(1) << bits;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  auto bucket = [&](int64_t r) -> int64_t {
    uint64_t k[NW];
    k[0] = __ldg(k0 + r);
    if constexpr (NW == 2) k[1] = __ldg(k1 + r);
    return static_cast<int64_t>(bucket_of(hash_key<NW>(k), bits));
  };
  // offsets[b] = first row whose bucket is >= b (n for b = P): the rows are
  // in bucket order, so a lower-bound search per bucket (~log2 n probes)
  // replaces reading every row
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b <= P; b += stride) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = lo + ((hi - lo) >> 1);
      if (bucket(mid) < b) lo = mid + 1;
      else hi = mid;
    }
    offsets[b] = static_cast<uint32_t>(lo);
  }
}
}  // namespace

cudaError_t launch_part_bounds(int nwords, const uint64_t* const* keys, const uint32_t* n_rows, int bits,
                               uint32_t* offsets, int num_sms, cudaStream_t st)
{
  const int grid = static_cast<int>(std::min<int64_t>(((int64_t(1) << bits) + 256) / 256, int64_t(num_sms) * 8));
  if (nwords == 1) k_part_bounds<1><<<grid, 256, 0, st>>>(keys[0], nullptr, n_rows, bits, offsets);
  else k_part_bounds<2><<<grid, 256, 0, st>>>(keys[0], keys[1], n_rows, bits, offsets);
  return cudaGetLastError();
}

cudaError_t launch_part_items(const PartPlan& pp, int64_t n, int num_sms, cudaStream_t st)
{
  (void)n;
  k_part_items<<<grid_rows(int64_t(1) << pp.bits, 256, num_sms * 8), 256, 0, st>>>(pp);
  return cudaGetLastError();
}

cudaError_t launch_part_scatter(const Plan& p, int64_t n, const PartPlan& pp, const PartBufs& out, int num_sms,
                                cudaStream_t st)
{
  const int grid = grid_rows(n, 256, num_sms * 8);
  if (p.key.nwords == 1) k_part_scatter<1><<<grid, 256, 0, st>>>(p, n, pp, out);
  else k_part_scatter<2><<<grid, 256, 0, st>>>(p, n, pp, out);
  return cudaGetLastError();
}

namespace {
cudaError_t launch_folds(const Plan& p, const PartPlan& pp, const PartBufs& sorted, const OutPlan& op, int num_sms,
                         cudaStream_t st);

template <int NW, int NCH>
cudaError_t launch_part_agg_impl(const Plan& p, const PartPlan& pp, const PartBufs& in, const TableRef& t,
                                 const SmemLayout& sl, int num_sms, cudaStream_t st)
{
  const int block   = 256;
  const int warps   = block / 32;
  const size_t smem = static_cast<size_t>(sl.total) * warps;
  cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_part_agg<NW, NCH>), smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e          = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_part_agg<NW, NCH>, block, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  k_part_agg<NW, NCH><<<num_sms * per_sm, block, smem, st>>>(p, pp, in, t, sl);
  return cudaGetLastError();
}

template <int NW>
cudaError_t launch_part_agg_nw(const Plan& p, const PartPlan& pp, const PartBufs& in, const TableRef& t,
                               const SmemLayout& sl, int num_sms, cudaStream_t st)
{
  if (p.nchan <= 2) return launch_part_agg_impl<NW, 2>(p, pp, in, t, sl, num_sms, st);
  if (p.nchan <= 4) return launch_part_agg_impl<NW, 4>(p, pp, in, t, sl, num_sms, st);
  return launch_part_agg_impl<NW, kMaxChannels>(p, pp, in, t, sl, num_sms, st);
}

// Shared memory of k_part_ranked: eight warps per CTA, each with its table,
// list and as many rank records as fit the CTA's share of the SM's shared
// memory (kRankedCtasPerSm CTAs per SM); buckets with more rows keep their
// records in global memory.
template <int NW>
cudaError_t launch_part_ranked_nw(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                                  uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st)
{
  const int block = 256;
  const int warps = block / 32;
  int dev = 0, per_sm_bytes = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
    return e;
  SmemLayout sl{};
  sl.slots    = S;
  sl.keys_off = 0;
  sl.rows_off = (S + 1) * NW * 8;
  sl.total    = (sl.rows_off + (S + 1) * 4 + 15) & ~15u;
  RankedLayout rl{};
  rl.scratch_off = sl.total;
  rl.rec_off     = (rl.scratch_off + (S + 32) * 4 + 15) & ~15u;
  // per CTA: its share of the SM less reserved and static memory
  const int64_t cta_bytes = per_sm_bytes / kRankedCtasPerSm - 2048;
  const int64_t rec_bytes = cta_bytes / warps - rl.rec_off;
  rl.rec_rows = rec_bytes > 0 ? static_cast<uint32_t>(std::min<int64_t>(rec_bytes / 4, pp.slice_rows)) & ~31u : 0u;
  rl.stride   = (rl.rec_off + rl.rec_rows * 4 + 15) & ~15u;
  const size_t smem = static_cast<size_t>(rl.stride) * warps;
  if ((e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_part_ranked<NW>), smem)) != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_part_ranked<NW>, block, smem)) != cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  k_part_ranked<NW><<<num_sms * per_sm, block, smem, st>>>(p, pp, in, sorted, sl, rl, op);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return launch_folds(p, pp, sorted, op, num_sms, st);
}

// Shared memory of k_part_ranked_cta: the table, counters and list, and as
// many rank records as leave room for up to four CTAs per SM (at least 2,048
// records each); buckets with more rows keep their records in global memory.
template <int NW>
cudaError_t launch_part_ranked_cta_nw(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                                      uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st)
{
  if (S < static_cast<uint32_t>(kCtaRankThreads) || S > 4096 || (S & (S - 1)) != 0 || pp.slice_rows > kCtaMaxSliceRows)
    return cudaErrorInvalidValue;
  int dev = 0, per_sm_bytes = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
    return e;
  CtaRankLayout cl{};
  cl.slots    = S;
  cl.cnt_off  = ((S + 1) * NW * 8 + 15) & ~15u;
  cl.list_off = (cl.cnt_off + (S + 2) * 4 + 15) & ~15u;
  cl.rec_off  = (cl.list_off + (S + 1) * 4 + 15) & ~15u;
  int ctas    = 4;
  while (ctas > 1 && static_cast<int64_t>(per_sm_bytes) / ctas - 2048 < cl.rec_off + 2048 * 4) --ctas;
  const int64_t rec_bytes = static_cast<int64_t>(per_sm_bytes) / ctas - 2048 - cl.rec_off;
  cl.rec_rows = rec_bytes > 0 ? static_cast<uint32_t>(std::min<int64_t>(rec_bytes / 4, pp.slice_rows)) & ~31u : 0u;
  cl.total    = (cl.rec_off + cl.rec_rows * 4 + 15) & ~15u;
  if ((e = ensure_dynamic_smem(reinterpret_cast<const void*>(k_part_ranked_cta<NW>), cl.total)) != cudaSuccess)
    return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_part_ranked_cta<NW>, kCtaRankThreads,
                                                         cl.total)) != cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  k_part_ranked_cta<NW><<<num_sms * per_sm, kCtaRankThreads, cl.total, st>>>(p, pp, in, sorted, cl, op);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return launch_folds(p, pp, sorted, op, num_sms, st);
}
}  // namespace

cudaError_t launch_part_ranked_cta(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                                   uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st)
{
  return p.key.nwords == 1 ? launch_part_ranked_cta_nw<1>(p, pp, in, sorted, S, op, num_sms, st)
                           : launch_part_ranked_cta_nw<2>(p, pp, in, sorted, S, op, num_sms, st);
}

namespace {
// One k_part_fold launch per value channel, each on its physical type.
cudaError_t launch_folds(const Plan& p, const PartPlan& pp, const PartBufs& sorted, const OutPlan& op, int num_sms,
                         cudaStream_t st)
{
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < p.nchan; ++c) {
    switch (p.chan[c].ptype) {
      case P_I8: e = launch_fold<P_I8>(p, pp, sorted, op, c, num_sms, st); break;
      case P_I16: e = launch_fold<P_I16>(p, pp, sorted, op, c, num_sms, st); break;
      case P_I32: e = launch_fold<P_I32>(p, pp, sorted, op, c, num_sms, st); break;
      case P_I64: e = launch_fold<P_I64>(p, pp, sorted, op, c, num_sms, st); break;
      case P_U8: e = launch_fold<P_U8>(p, pp, sorted, op, c, num_sms, st); break;
      case P_U16: e = launch_fold<P_U16>(p, pp, sorted, op, c, num_sms, st); break;
      case P_U32: e = launch_fold<P_U32>(p, pp, sorted, op, c, num_sms, st); break;
      case P_U64: e = launch_fold<P_U64>(p, pp, sorted, op, c, num_sms, st); break;
      case P_F32: e = launch_fold<P_F32>(p, pp, sorted, op, c, num_sms, st); break;
      case P_F64: e = launch_fold<P_F64>(p, pp, sorted, op, c, num_sms, st); break;
      default: e = launch_fold<P_BOOL>(p, pp, sorted, op, c, num_sms, st); break;
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace

cudaError_t launch_part_ranked(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                               uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st)
{
  return p.key.nwords == 1 ? launch_part_ranked_nw<1>(p, pp, in, sorted, S, op, num_sms, st)
                           : launch_part_ranked_nw<2>(p, pp, in, sorted, S, op, num_sms, st);
}

cudaError_t launch_part_agg(const Plan& p, const PartPlan& pp, const PartBufs& in, const TableRef& t,
                            const SmemLayout& sl, int num_sms, cudaStream_t st)
{
  return p.key.nwords == 1 ? launch_part_agg_nw<1>(p, pp, in, t, sl, num_sms, st)
                           : launch_part_agg_nw<2>(p, pp, in, t, sl, num_sms, st);
}

cudaError_t launch_part_region_finalize(const Plan& p, const PartPlan& pp, const TableRef& t, const OutPlan& op,
                                       int num_sms, cudaStream_t st)
{
  const int grid = grid_rows(static_cast<int64_t>(t.cap + 1), 256, num_sms * 8);
  if (p.key.nwords == 1) k_part_region_finalize<1><<<grid, 256, 0, st>>>(p, pp, t, op);
  else k_part_region_finalize<2><<<grid, 256, 0, st>>>(p, pp, t, op);
  return cudaGetLastError();
}

}  // namespace gbx
