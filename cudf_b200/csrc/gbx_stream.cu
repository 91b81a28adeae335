// gbx_stream.cu -- the low-cardinality plain path: each CTA streams tiles of
// the caller's rows through shared memory and groups every tile before it
// touches its table.
//
// Per tile of kSTile rows (kSPer rows a thread, strided so that every load
// instruction of a warp is one contiguous run):
//   1. each row's packed key finds (or takes) its slot in the CTA's table
//      (open addressing in shared memory) and its rank among the tile's rows
//      of that slot (one 32-bit shared atomic);
//   2. one block scan turns the slots' row counts into the first position of
//      each slot's run;
//   3. each channel's values are loaded and stored at their row's position,
//      so the tile's values lie in shared memory group by group;
//   4. the runs are cut into chunks of at most kSChunk rows; each thread
//      folds one chunk in registers (the fold of chan_acc_add, specialised
//      on the channel's physical type) and merges it into its slot with
//      shared reductions.  A warp whose 32 chunks all belong to one group
//      (a group of thousands of rows in the tile) first combines them with
//      shuffles and merges once: 64-bit shared reductions that many lanes
//      aim at one address at once serialise.  A chunk's VAR sums are
//      relative to its own shift (its first value); merges re-centre them.
// After its last tile the CTA merges its table into the global one.
//
// This replaces the reference's per-row find-or-insert into a cuco set plus
// per-row atomics on sparse result columns (cpp/src/groupby/hash/groupby.cu:
// 548-622, groupby_kernels.cuh:98-105, aggregation.cuh:558-573) for inputs
// whose groups fit a CTA table.  Every loop is bounded: probes by
// `smem_probes` (then the row goes to the global table directly), CAS loops
// by their spin limit.
#include <algorithm>

#include "gbx_kernels.hpp"
#include "gbx_warpcore.cuh"

namespace gbx {

using namespace dev;

namespace {

constexpr int kSBlock          = 512;
constexpr int kSPer            = 8;
constexpr int kSTile           = kSBlock * kSPer;
constexpr uint32_t kSNoRec     = 0xffffffffu;
constexpr int kSMaxSlots       = 4096;
constexpr int kSChunk          = 32;  // rows of one group folded by one thread
constexpr size_t kSSmemBudget1 = 220 * 1024;  // one CTA an SM

// Dynamic shared memory after the table (SmemLayout at offset 0): each
// slot's first position and first chunk (S + 2 words each), then per
// channel kSTile value words and kSTile validity bytes.
struct StreamLayout {
  uint32_t off_off;
  uint32_t coff_off;
  uint32_t spill_off;  // kSTile u16: tile rows whose key found no slot
  uint32_t vals_off;
  uint32_t valid_off;
  uint32_t total;
};

StreamLayout stream_layout(const SmemLayout& sl, int nchan)
{
  StreamLayout ly{};
  uint32_t o  = sl.total;
  ly.off_off  = o;
  o += (sl.slots + 2) * 4;
  ly.coff_off = o;
  o += (sl.slots + 2) * 4;
  ly.spill_off = o;
  o += kSTile * 2;
  o           = (o + 15) & ~15u;
  ly.vals_off = o;
  o += static_cast<uint32_t>(nchan) * kSTile * 8;
  ly.valid_off = o;
  o += static_cast<uint32_t>(nchan) * kSTile;
  ly.total = (o + 15) & ~15u;
  return ly;
}

// Key of row r.  KM 0: the plan's packing (any key columns that fit one
// word); 1 / 2: one plain 8- / 4-byte integer key column without a mask,
// whose packed key is the column's bits.
template <int KM>
__device__ __forceinline__ bool stream_key(const KeyPlan& kp, int64_t r, uint64_t& k)
{
  if constexpr (KM == 1) {
    k = __ldg(reinterpret_cast<const unsigned long long*>(kp.cols[0].data) + kp.cols[0].offset + r);
    return true;
  } else if constexpr (KM == 2) {
    k = __ldg(reinterpret_cast<const uint32_t*>(kp.cols[0].data) + kp.cols[0].offset + r);
    return true;
  } else {
    uint64_t kk[1];
    const bool kept = pack_key<1>(kp, r, kk);
    k               = kk[0];
    return kept;
  }
}

// Value bits of channel c at row r (false: null, or a dictionary index out
// of range, which also sets S_BAD_INDEX).
__device__ __forceinline__ bool stream_value(const Channel& ch, int64_t r, uint64_t& b, int32_t* status)
{
  const int64_t i = r + ch.offset;
  if (!bit_valid(ch.mask, i)) return false;
  if (ch.dict_data == nullptr) {
    b = load_bits(ch.data, i, pt_width(ch.ptype));
    return true;
  }
  bool ok;
  b = value_bits(ch, r, ok);
  if (!ok) atomicOr(status, S_BAD_INDEX);
  return ok;
}

// Slot of key k in the CTA table (inserting it into an empty slot), or -1
// after `max_probes` slots.  Plain loads and atomicCAS (no volatile asm): the
// compiler may then keep a thread's row loads in flight across its probes.
// A stale read of an empty slot is harmless: the CAS then reports the key
// that won the slot.
__device__ __forceinline__ int64_t smem_find_or_insert(uint64_t* skeys, uint32_t mask, uint64_t k,
                                                       uint32_t max_probes)
{
  uint32_t s = static_cast<uint32_t>(fmix64(k)) & mask;
  for (uint32_t p = 0; p < max_probes; ++p) {
    const uint64_t cur = skeys[s];
    if (cur == k) return s;
    if (cur == kEmptyWord) {
      const unsigned long long old =
        atomicCAS(reinterpret_cast<unsigned long long*>(skeys + s), static_cast<unsigned long long>(kEmptyWord),
                  static_cast<unsigned long long>(k));
      if (old == kEmptyWord || old == k) return s;
    }
    s = (s + 1) & mask;
  }
  return -1;
}

// Merges a thread's partial accumulators A of one group into slot s of the
// CTA table.  The partial's VAR sums are relative to its own shift A.k; they
// are re-centred on the slot's shift Ks (recorded by the first merge):
// with d = A.k - Ks, sum (x-Ks)^2 = s2 + 2 d S1 + n d^2 and sum (x-Ks) = S1 + n d.
template <int PT>
__device__ __forceinline__ void merge_stream_partial(const Channel& ch, const ChanAcc& A, const Level<Shared>& L,
                                                     uint32_t s, int32_t* status)
{
  if (A.cnt == 0) return;
  constexpr bool kFloat = PT == P_F32 || PT == P_F64;
  constexpr bool kM64   = PT == P_I64 || PT == P_U64 || PT == P_F64;
  if (ch.a_cnt >= 0) Shared::add_u32(L.acc(ch.a_cnt) + s * 4, A.cnt);
  if (ch.a_min >= 0) {
    if (kM64) Shared::min_u64(L.acc(ch.a_min) + s * 8, A.mn);
    else Shared::min_u32(L.acc(ch.a_min) + s * 4, static_cast<uint32_t>(A.mn));
  }
  if (ch.a_max >= 0) {
    if (kM64) Shared::max_u64(L.acc(ch.a_max) + s * 8, A.mx);
    else Shared::max_u32(L.acc(ch.a_max) + s * 4, static_cast<uint32_t>(A.mx));
  }
  if (kFloat) {
    if (ch.a_sum >= 0) Shared::add_f64(L.acc(ch.a_sum) + s * 8, __longlong_as_double(static_cast<long long>(A.sum)));
    if (ch.a_sq >= 0) Shared::add_f64(L.acc(ch.a_sq) + s * 8, __longlong_as_double(static_cast<long long>(A.sq)));
    if (ch.a_prod >= 0)
      mul_cas_f64<Shared>(L.acc(ch.a_prod) + s * 8, __longlong_as_double(static_cast<long long>(A.prod)), status);
  } else {
    if (ch.a_sum >= 0) Shared::add_u64(L.acc(ch.a_sum) + s * 8, A.sum);
    if (ch.a_sq >= 0) Shared::add_u64(L.acc(ch.a_sq) + s * 8, A.sq);
    if (ch.a_prod >= 0) mul_cas_i64<Shared>(L.acc(ch.a_prod) + s * 8, static_cast<int64_t>(A.prod), status);
  }
  if (ch.a_k >= 0) {
    if (A.k == kShiftUnset) {
      // every valid value was NaN: the partial sums are NaN already
      Shared::add_f64(L.acc(ch.a_s2) + s * 8, A.s2);
      if (ch.a_s1 >= 0) Shared::add_f64(L.acc(ch.a_s1) + s * 8, A.s1);
    } else {
      const double Kp = __longlong_as_double(static_cast<long long>(A.k));
      const double Ks = get_shift<Shared>(L.acc(ch.a_k) + s * 8, Kp);
      const double S1 = shifted_sum(kFloat, PT, A.sum, static_cast<uint64_t>(__double_as_longlong(A.s1)), A.cnt, Kp);
      const double d  = Kp - Ks;
      const double n  = static_cast<double>(A.cnt);
      Shared::add_f64(L.acc(ch.a_s2) + s * 8, A.s2 + 2.0 * d * S1 + n * d * d);
      if (ch.a_s1 >= 0) Shared::add_f64(L.acc(ch.a_s1) + s * 8, S1 + n * d);
    }
  }
}

__device__ __forceinline__ uint64_t shfl_down_u64(uint64_t v, int o)
{
  return static_cast<uint64_t>(__shfl_down_sync(0xffffffffu, static_cast<unsigned long long>(v), o));
}

// The sum of every lane's partial in lane 0 (all 32 lanes call it), field
// by field so that few registers are live: the identities of chan_acc_init
// leave MIN/MAX/SUM unchanged by an empty partial; PRODUCT and the VAR sums
// look at the counts.
template <int PT>
__device__ __forceinline__ void warp_combine(uint32_t roles, ChanAcc& A)
{
  constexpr bool kFloat = PT == P_F32 || PT == P_F64;
  auto fadd = [](uint64_t a, uint64_t b) {
    return static_cast<uint64_t>(__double_as_longlong(__longlong_as_double(static_cast<long long>(a)) +
                                                      __longlong_as_double(static_cast<long long>(b))));
  };
#pragma unroll 1
  for (int o = 16; o > 0; o >>= 1) {
    const uint32_t nb = __shfl_down_sync(0xffffffffu, A.cnt, o);
    if (roles & R_MIN) A.mn = min(A.mn, shfl_down_u64(A.mn, o));
    if (roles & R_MAX) A.mx = max(A.mx, shfl_down_u64(A.mx, o));
    uint64_t sumb = 0;
    if (roles & (R_SUM | R_VAR)) sumb = shfl_down_u64(A.sum, o);
    if (roles & R_SQ) {
      const uint64_t v = shfl_down_u64(A.sq, o);
      A.sq             = kFloat ? fadd(A.sq, v) : A.sq + v;
    }
    if (roles & R_PROD) {
      const uint64_t v = shfl_down_u64(A.prod, o);
      if (nb != 0)
        A.prod = A.cnt == 0 ? v
                 : kFloat   ? static_cast<uint64_t>(__double_as_longlong(
                              __longlong_as_double(static_cast<long long>(A.prod)) *
                              __longlong_as_double(static_cast<long long>(v))))
                            : A.prod * v;
    }
    if (roles & R_VAR) {
      const uint64_t kb = shfl_down_u64(A.k, o);
      const double s2b  = __shfl_down_sync(0xffffffffu, A.s2, o);
      const double s1b  = __shfl_down_sync(0xffffffffu, A.s1, o);
      if (nb != 0) {
        if (A.cnt == 0) {
          A.k  = kb;
          A.s2 = s2b;
          A.s1 = s1b;
        } else if (A.k == kShiftUnset || kb == kShiftUnset) {
          if (A.k == kShiftUnset) A.k = kb;
          A.s2 += s2b;
          A.s1 += s1b;
        } else {
          const double Ka = __longlong_as_double(static_cast<long long>(A.k));
          const double Kb = __longlong_as_double(static_cast<long long>(kb));
          const double S1 = shifted_sum(kFloat, PT, sumb, static_cast<uint64_t>(__double_as_longlong(s1b)), nb, Kb);
          const double d  = Kb - Ka;
          const double n  = static_cast<double>(nb);
          A.s2 += s2b + 2.0 * d * S1 + n * d * d;
          if (kFloat) A.s1 += S1 + n * d;
        }
      }
    }
    if (roles & (R_SUM | R_VAR)) A.sum = kFloat ? fadd(A.sum, sumb) : A.sum + sumb;
    A.cnt += nb;
  }
}

// Folds staged positions [p0, p1) (one chunk of one group) of a channel and
// merges the result into slot s; `uniform`: the warp's 32 chunks are all of
// slot s, so they are combined with shuffles and lane 0 merges once.
template <int PT>
__device__ __forceinline__ void fold_chunk_merge(const Channel& ch, const uint64_t* vals, const uint8_t* valid,
                                                 uint32_t p0, uint32_t p1, uint32_t s, bool uniform,
                                                 const Level<Shared>& L, int32_t* status)
{
  const uint32_t roles = chan_roles(ch);
  ChanAcc A;
  chan_acc_init(A);
  for (uint32_t p = p0; p < p1; ++p)
    if (valid[p]) chan_acc_add<PT>(ch, roles, A, vals[p]);
  if (uniform) {
    warp_combine<PT>(roles, A);
    if ((threadIdx.x & 31) == 0) merge_stream_partial<PT>(ch, A, L, s, status);
  } else {
    merge_stream_partial<PT>(ch, A, L, s, status);
  }
}

template <int KM>
__global__ void __launch_bounds__(kSBlock, 2) k_agg_stream(const __grid_constant__ Plan plan,
                                                        const __grid_constant__ TableRef t,
                                                        const __grid_constant__ SmemLayout sl,
                                                        const __grid_constant__ StreamLayout ly, int64_t n,
                                                        uint32_t smem_probes, uint32_t max_probes)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t warp_sums[kSBlock / 32];
  __shared__ uint32_t s_special;
  __shared__ uint32_t s_nspill;
  const uint32_t S    = sl.slots;
  uint64_t* skeys     = reinterpret_cast<uint64_t*>(smem + sl.keys_off);
  uint32_t* srows     = reinterpret_cast<uint32_t*>(smem + sl.rows_off);
  uint32_t* off       = reinterpret_cast<uint32_t*>(smem + ly.off_off);
  uint32_t* coff      = reinterpret_cast<uint32_t*>(smem + ly.coff_off);
  uint16_t* spill     = reinterpret_cast<uint16_t*>(smem + ly.spill_off);
  uint64_t* vals      = reinterpret_cast<uint64_t*>(smem + ly.vals_off);
  uint8_t* valid      = smem + ly.valid_off;
  const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int lane      = threadIdx.x & 31;
  const int warp      = threadIdx.x >> 5;

  // identity fill; per-slot counts zeroed
  for (uint32_t s = threadIdx.x; s <= S; s += kSBlock) {
    skeys[s] = kEmptyWord;
    srows[s] = 0;
    off[s]   = 0;
    for (int a = 0; a < plan.acc.nacc; ++a) {
      const uint64_t id = identity_bits(plan.acc.kind[a]);
      if (acc_bytes(plan.acc.kind[a]) == 4) reinterpret_cast<uint32_t*>(smem + sl.acc_off[a])[s] = static_cast<uint32_t>(id);
      else reinterpret_cast<uint64_t*>(smem + sl.acc_off[a])[s] = id;
    }
  }
  if (threadIdx.x == 0) {
    s_special   = 0;
    s_nspill    = 0;
    off[S + 1]  = 0;
    coff[S + 1] = 0;
  }
  __syncthreads();

  const Level<Shared> L{base, &sl};
  const Level<Global> G = global_level(t);
  const int64_t ntiles  = (n + kSTile - 1) / kSTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t t0 = tile * kSTile;
    // 1. slot and rank of each of this thread's rows (off[] counts the rows)
    uint64_t k[kSPer];
    bool kept[kSPer];
#pragma unroll
    for (int q = 0; q < kSPer; ++q) {
      const int64_t r = t0 + threadIdx.x + q * kSBlock;
      kept[q]         = r < n && stream_key<KM>(plan.key, r, k[q]);
    }
    uint32_t rec[kSPer];
#pragma unroll
    for (int q = 0; q < kSPer; ++q) {
      rec[q]        = kSNoRec;
      bool to_spill = false;
      if (kept[q]) {
        int64_t s;
        if (k[q] == kEmptyWord) {
          s = S;
          if (s_special == 0) s_special = 1;
        } else {
          s = smem_find_or_insert(skeys, S - 1, k[q], smem_probes);
        }
        if (s >= 0) rec[q] = static_cast<uint32_t>(s) << 16;
        else to_spill = true;
      }
      // rows whose key found no slot in the CTA table are listed and sent to
      // the global table below by all threads together (one lane per row
      // would run the global path with most of the warp idle)
      const uint32_t bal = __ballot_sync(0xffffffffu, to_spill);
      if (bal != 0) {
        uint32_t sb = 0;
        if (lane == 0) sb = atomicAdd(&s_nspill, static_cast<uint32_t>(__popc(bal)));
        sb = __shfl_sync(0xffffffffu, sb, 0);
        if (to_spill)
          spill[sb + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint16_t>(threadIdx.x + q * kSBlock);
      }
    }
    // ranks: the lanes of a warp that share a slot take consecutive ranks
    // from one shared atomic (a few hot groups would otherwise serialise)
#pragma unroll
    for (int q = 0; q < kSPer; ++q) {
      const bool has    = rec[q] != kSNoRec;
      const uint32_t sk = has ? (rec[q] >> 16) : 0xffffffffu;
      const uint32_t pe = __match_any_sync(0xffffffffu, sk);
      const int leader  = __ffs(pe) - 1;
      uint32_t b        = 0;
      if (has && lane == leader) b = atomicAdd(off + sk, static_cast<uint32_t>(__popc(pe)));
      b = __shfl_sync(0xffffffffu, b, leader);
      if (has) rec[q] |= b + static_cast<uint32_t>(__popc(pe & ((1u << lane) - 1u)));
    }
    __syncthreads();
    // 1b. the listed rows update the global table directly
    {
      const uint32_t nsp = s_nspill;
      for (uint32_t i = threadIdx.x; i < nsp; i += kSBlock) {
        const int64_t r = t0 + spill[i];
        uint64_t kk[1];
        stream_key<KM>(plan.key, r, kk[0]);
        const int64_t g = global_slot<1>(t, kk, max_probes);
        if (g >= 0) accumulate_row<Global>(plan, G, g, r, t.status);
      }
    }
    // 2. row counts -> first position of each slot's run (exclusive scan over
    //    S + 1 slots, kScanPer per thread); COUNT_ALL rows added per slot
    {
      constexpr int kPerMax = (kSMaxSlots + 1 + kSBlock - 1) / kSBlock;
      const int per         = static_cast<int>((S + 1 + kSBlock - 1) / kSBlock);
      uint32_t c[kPerMax];
      uint32_t sum = 0;
#pragma unroll
      for (int q = 0; q < kPerMax; ++q) {
        // rows in the low half, chunks of at most kSChunk rows in the high half
        const uint32_t s  = threadIdx.x * per + q;
        const uint32_t rw = (q < per && s <= S) ? off[s] : 0u;
        c[q]              = rw | (((rw + kSChunk - 1) / kSChunk) << 16);
        sum += c[q];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
      }
      if (lane == 31) warp_sums[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        const uint32_t w = lane < kSBlock / 32 ? warp_sums[lane] : 0u;
        uint32_t wi      = w;
#pragma unroll
        for (int d = 1; d < kSBlock / 32; d <<= 1) {
          const uint32_t o = __shfl_up_sync(0xffffffffu, wi, d);
          if (lane >= d) wi += o;
        }
        if (lane < kSBlock / 32) warp_sums[lane] = wi - w;
        if (lane == kSBlock / 32 - 1) {
          off[S + 1]  = wi & 0xffffu;
          coff[S + 1] = wi >> 16;
        }
      }
      __syncthreads();
      uint32_t run = warp_sums[warp] + incl - sum;
#pragma unroll
      for (int q = 0; q < kPerMax; ++q) {
        const uint32_t s = threadIdx.x * per + q;
        if (q < per && s <= S) {
          off[s]  = run & 0xffffu;
          coff[s] = run >> 16;
          srows[s] += c[q] & 0xffffu;
          run += c[q];
        }
      }
    }
    __syncthreads();
    // 3. each channel's values at their row's position
    for (int ch = 0; ch < plan.nchan; ++ch) {
      const Channel& chan = plan.chan[ch];
      uint64_t b[kSPer];
      bool v[kSPer];
#pragma unroll
      for (int q = 0; q < kSPer; ++q) {
        b[q] = 0;
        v[q] = rec[q] != kSNoRec && stream_value(chan, t0 + threadIdx.x + q * kSBlock, b[q], t.status);
      }
      uint64_t* cv = vals + static_cast<size_t>(ch) * kSTile;
      uint8_t* cvv = valid + static_cast<size_t>(ch) * kSTile;
#pragma unroll
      for (int q = 0; q < kSPer; ++q) {
        if (rec[q] == kSNoRec) continue;
        const uint32_t p = off[rec[q] >> 16] + (rec[q] & 0xffffu);
        cv[p]            = b[q];
        cvv[p]           = v[q] ? 1 : 0;
      }
    }
    __syncthreads();
    // 4. one chunk (<= kSChunk rows of one group) per thread; warps whose
    //    chunks are all of one group combine them before merging
    const uint32_t nchunks = coff[S + 1];
    for (uint32_t c0 = static_cast<uint32_t>(warp) * 32; c0 < nchunks; c0 += kSBlock) {
      const uint32_t ci  = c0 + lane;
      const bool active  = ci < nchunks;
      uint32_t s = 0, p0 = 0, p1 = 0;
      if (active) {
        // the chunk's slot: the last slot whose chunks start at or before it
        uint32_t lo = 0, hi = S;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (coff[mid] <= ci) lo = mid;
          else hi = mid - 1;
        }
        s  = lo;
        p0 = off[s] + (ci - coff[s]) * kSChunk;
        p1 = min(p0 + kSChunk, off[s + 1]);
      }
      // every lane takes part in both warp operations (an inactive lane
      // must not skip the shuffle, or the warp waits for it forever)
      const uint32_t s_lane0 = __shfl_sync(0xffffffffu, s, 0);
      const bool uniform     = __all_sync(0xffffffffu, active && s == s_lane0);
      if (!active) continue;
      for (int ch = 0; ch < plan.nchan; ++ch) {
        const Channel& chan = plan.chan[ch];
        const uint64_t* cv  = vals + static_cast<size_t>(ch) * kSTile;
        const uint8_t* cvv  = valid + static_cast<size_t>(ch) * kSTile;
#define GBX_FOLD_CHUNK(P) fold_chunk_merge<P>(chan, cv, cvv, p0, p1, s, uniform, L, t.status)
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
      }
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s <= S; s += kSBlock) off[s] = 0;
    if (threadIdx.x == 0) s_nspill = 0;
    __syncthreads();
  }

  // merge the CTA's table into the global one
  for (uint32_t s = threadIdx.x; s <= S; s += kSBlock) {
    const uint64_t k1[1] = {skeys[s]};
    const bool occupied  = (s < S) ? k1[0] != kEmptyWord : (s_special != 0);
    if (!occupied || srows[s] == 0) continue;
    const int64_t g = global_slot<1>(t, k1, max_probes);
    if (g >= 0) merge_slot<Shared>(plan, L, s, G, g, t.status);
  }
}

template <int KM>
cudaError_t launch_stream_km(const Plan& p, const TableRef& t, const SmemLayout& sl, const StreamLayout& ly,
                             int64_t n, int num_sms, uint32_t smem_probes, uint32_t max_probes, cudaStream_t st)
{
  const void* fn = reinterpret_cast<const void*>(k_agg_stream<KM>);
  cudaError_t e  = ensure_dynamic_smem(fn, ly.total);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_agg_stream<KM>, kSBlock, ly.total)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int64_t ntiles = (n + kSTile - 1) / kSTile;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(num_sms) * per_sm)));
  k_agg_stream<KM><<<grid, kSBlock, ly.total, st>>>(p, t, sl, ly, n, smem_probes, max_probes);
  return cudaGetLastError();
}

// Key mode of a plan (see stream_key).
int stream_key_mode(const KeyPlan& kp)
{
  if (kp.ncols == 1) {
    const KeyCol& kc = kp.cols[0];
    if (kc.mask == nullptr && !kc.is_float && !kc.is_bool && !kc.null_bit && kc.shift == 0 && kc.word == 0) {
      if (kc.width == 8) return 1;
      if (kc.width == 4) return 2;
    }
  }
  return 0;
}

}  // namespace

bool stream_fits(const Plan& p, const SmemLayout& sl)
{
  if (p.key.nwords != 1 || plan_has_arg(p) || sl.slots > static_cast<uint32_t>(kSMaxSlots)) return false;
  return stream_layout(sl, p.nchan).total <= kSSmemBudget1;
}

size_t stream_smem_bytes(const Plan& p, const SmemLayout& sl) { return stream_layout(sl, p.nchan).total; }

cudaError_t launch_agg_stream(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                              uint32_t smem_probes, uint32_t max_probes, cudaStream_t st)
{
  if (!stream_fits(p, sl)) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  const StreamLayout ly = stream_layout(sl, p.nchan);
  switch (stream_key_mode(p.key)) {
    case 1: return launch_stream_km<1>(p, t, sl, ly, n, num_sms, smem_probes, max_probes, st);
    case 2: return launch_stream_km<2>(p, t, sl, ly, n, num_sms, smem_probes, max_probes, st);
    default: return launch_stream_km<0>(p, t, sl, ly, n, num_sms, smem_probes, max_probes, st);
  }
}

}  // namespace gbx
