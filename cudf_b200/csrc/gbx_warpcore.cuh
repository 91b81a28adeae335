// gbx_warpcore.cuh -- the warp-exclusive table core shared by the warp-private
// kernel (gbx_warp.cu) and the partitioned kernel (gbx_part.cu).
//
// A warp owns a shared-memory table nobody else touches.  For each batch of
// up to 32 rows it
//   1. finds or inserts each key: lanes probe in parallel; missing keys are
//      inserted in rounds where, for every contended empty slot, one lane
//      (__match_any_sync on the target slot) writes its key and the others
//      re-probe -- so distinct keys with distinct targets insert together;
//   2. ranks lanes that hit the same slot (__match_any_sync) and applies the
//      rows in rounds, one row per slot per round, with plain loads and
//      stores (no atomics).
#pragma once

#include "gbx_kernels.hpp"
#include "gbx_table.cuh"

namespace gbx {
namespace dev {

constexpr uint32_t kFull = 0xffffffffu;

// ------------------------------------------------------------- row sources

// (RowSource, the caller's columns, is in gbx_table.cuh.)

// Rows of the radix-partitioned copies (keys already packed, dictionary
// values resolved, validity as one byte per row).
struct PartSource {
  const PartBufs* pb;
  template <int NW>
  __device__ __forceinline__ bool key(int64_t r, uint64_t (&k)[NW]) const
  {
#pragma unroll
    for (int w = 0; w < NW; ++w) k[w] = __ldg(pb->keys[w] + r);
    return true;
  }
  __device__ __forceinline__ bool value(int c, int64_t r, uint64_t& b, int32_t*) const
  {
    const PartCol& pc = pb->col[c];
    if (pc.valid != nullptr && __ldg(pc.valid + r) == 0) return false;
    b = load_bits(pc.vals, r, pc.width);
    return true;
  }
};

// ------------------------------------------------------- per-row values

// One lane's row: the raw value bits of each of up to NCH channels
// (dictionary resolved) and a validity bit per channel.  Loaded for a whole batch before probing so
// that the loads of all columns are in flight together.
template <int NCH>
struct RowVals {
  uint64_t bits[NCH];
  uint32_t valid;
};

template <int NCH, class Src>
__device__ __forceinline__ void load_row_values(const Plan& plan, const Src& src, bool act, int64_t r,
                                                RowVals<NCH>& v, int32_t* status)
{
  v.valid = 0;
#pragma unroll
  for (int c = 0; c < NCH; ++c) {
    v.bits[c] = 0;
    if (c < plan.nchan && act && src.value(c, r, v.bits[c], status)) v.valid |= 1u << c;
  }
}

// Applies one row to an exclusively owned shared-memory slot with plain
// loads and stores (aggregate_row, detail/aggregation/aggregation.cuh:558-573,
// with update_target_element's null skipping, :116-491).
template <int NCH>
__device__ __forceinline__ void apply_row(const Plan& plan, unsigned char* tb, const SmemLayout& sl, uint32_t s,
                                          const RowVals<NCH>& v)
{
  reinterpret_cast<uint32_t*>(tb + sl.rows_off)[s] += 1;
#pragma unroll
  for (int c = 0; c < NCH; ++c) {
    if (c >= plan.nchan) break;
    if (!((v.valid >> c) & 1u)) continue;
    const Channel& ch = plan.chan[c];
    const uint64_t b  = v.bits[c];
    if (ch.a_cnt >= 0) reinterpret_cast<uint32_t*>(tb + sl.acc_off[ch.a_cnt])[s] += 1;
    const bool m64 = minmax_is64(ch.ptype);
    if (ch.a_min >= 0) {
      const uint64_t e = enc_minmax(b, ch.ptype, true);
      if (m64) {
        uint64_t* p = reinterpret_cast<uint64_t*>(tb + sl.acc_off[ch.a_min]) + s;
        *p          = min(*p, e);
      } else {
        uint32_t* p = reinterpret_cast<uint32_t*>(tb + sl.acc_off[ch.a_min]) + s;
        *p          = min(*p, static_cast<uint32_t>(e));
      }
    }
    if (ch.a_max >= 0) {
      const uint64_t e = enc_minmax(b, ch.ptype, false);
      if (m64) {
        uint64_t* p = reinterpret_cast<uint64_t*>(tb + sl.acc_off[ch.a_max]) + s;
        *p          = max(*p, e);
      } else {
        uint32_t* p = reinterpret_cast<uint32_t*>(tb + sl.acc_off[ch.a_max]) + s;
        *p          = max(*p, static_cast<uint32_t>(e));
      }
    }
    double xf;
    if (ch.is_float) {
      xf = as_f64(b, ch.ptype);
      if (ch.a_sum >= 0) reinterpret_cast<double*>(tb + sl.acc_off[ch.a_sum])[s] += xf;
      if (ch.a_sq >= 0) reinterpret_cast<double*>(tb + sl.acc_off[ch.a_sq])[s] += xf * xf;
      if (ch.a_prod >= 0) reinterpret_cast<double*>(tb + sl.acc_off[ch.a_prod])[s] *= xf;
    } else {
      const int64_t x = as_i64(b, ch.ptype);
      if (ch.a_sum >= 0) reinterpret_cast<uint64_t*>(tb + sl.acc_off[ch.a_sum])[s] += static_cast<uint64_t>(x);
      if (ch.a_sq >= 0)
        reinterpret_cast<uint64_t*>(tb + sl.acc_off[ch.a_sq])[s] +=
          static_cast<uint64_t>(x) * static_cast<uint64_t>(x);
      if (ch.a_prod >= 0) {
        int64_t* p = reinterpret_cast<int64_t*>(tb + sl.acc_off[ch.a_prod]) + s;
        *p         = static_cast<int64_t>(static_cast<uint64_t>(*p) * static_cast<uint64_t>(x));
      }
      xf = (ch.ptype == P_U64) ? static_cast<double>(static_cast<uint64_t>(x)) : static_cast<double>(x);
    }
    if (ch.a_k >= 0) {
      // first non-NaN value becomes the shift; with no shift yet K is a NaN
      // pattern, so an all-NaN group's square sum is NaN
      uint64_t* kp = reinterpret_cast<uint64_t*>(tb + sl.acc_off[ch.a_k]) + s;
      if (*kp == kShiftUnset && !(xf != xf)) *kp = static_cast<uint64_t>(__double_as_longlong(xf));
      const double d = xf - __longlong_as_double(static_cast<long long>(*kp));
      reinterpret_cast<double*>(tb + sl.acc_off[ch.a_s2])[s] += d * d;
      if (ch.a_s1 >= 0) reinterpret_cast<double*>(tb + sl.acc_off[ch.a_s1])[s] += d;
    }
  }
}

// ------------------------------------------------------ the warp's table

// One warp's table in shared memory: S slots plus the reserved slot S.
template <int NW>
struct WarpTable {
  unsigned char* tb;
  const SmemLayout* sl;
  uint32_t S;
  __device__ __forceinline__ uint64_t* keys() const { return reinterpret_cast<uint64_t*>(tb + sl->keys_off); }
  __device__ __forceinline__ uint32_t* rows() const { return reinterpret_cast<uint32_t*>(tb + sl->rows_off); }

  // Empties the table: every key word empty and every accumulator of every
  // slot (the reserved slot S included) at its identity, so that inserting a
  // key only writes the key.  One accumulator array at a time, the lanes
  // taking consecutive slots.
  __device__ __forceinline__ void init(const AccLayout& al, int lane) const
  {
    uint64_t* kk = keys();
    uint32_t* rr = rows();
    for (uint32_t s = lane; s <= S; s += 32) {  // slot S keeps the all-ones key it stands for
#pragma unroll
      for (int w = 0; w < NW; ++w) kk[s * NW + w] = kEmptyWord;
      rr[s] = 0;
    }
    for (int a = 0; a < al.nacc; ++a) {
      const uint64_t id = identity_bits(al.kind[a]);
      if (acc_bytes(al.kind[a]) == 4) {
        uint32_t* p = reinterpret_cast<uint32_t*>(tb + sl->acc_off[a]);
        for (uint32_t s = lane; s <= S; s += 32) p[s] = static_cast<uint32_t>(id);
      } else {
        uint64_t* p = reinterpret_cast<uint64_t*>(tb + sl->acc_off[a]);
        for (uint32_t s = lane; s <= S; s += 32) p[s] = id;
      }
    }
    __syncwarp();
  }
  __device__ __forceinline__ void reset(const AccLayout& al, int lane) const { init(al, lane); }
  // Empties the keys and zeroes the row counts only (a table used to rank
  // rows by group, whose accumulators are not read).
  __device__ __forceinline__ void reset_keys(int lane) const
  {
    uint64_t* kk = keys();
    uint32_t* rr = rows();
    for (uint32_t s = lane; s <= S; s += 32) {
#pragma unroll
      for (int w = 0; w < NW; ++w) kk[s * NW + w] = kEmptyWord;
      rr[s] = 0;
    }
    __syncwarp();
  }
};

enum RowState { ST_DONE = 0, ST_PROBING = 1, ST_INSERT = 2, ST_FOUND = 3, ST_SPILL = 4 };

// Finds or inserts each active lane's key (warp-synchronous; all 32 lanes
// call it).  On return state is ST_FOUND (slot set; S for the all-ones key),
// ST_SPILL (the table is full around the key) or ST_DONE (inactive lane).
template <int NW>
__device__ __forceinline__ int warp_find_or_insert(const WarpTable<NW>& T, const AccLayout& al, bool act,
                                                   const uint64_t (&k)[NW], int lane, uint32_t& slot)
{
  uint64_t* keys       = T.keys();
  const uint32_t S     = T.S;
  const uint32_t smask = S - 1;
  int state            = ST_DONE;
  slot                 = 0;
  if (act) {
    if (key_is_empty<NW>(k)) {
      state = ST_FOUND;
      slot  = S;
    } else {
      state = ST_PROBING;
      slot  = static_cast<uint32_t>(hash_key<NW>(k)) & smask;
    }
  }
  // probe (the table only changes in the insertion rounds below)
  for (uint32_t p = 0; p <= S && __any_sync(kFull, state == ST_PROBING); ++p) {
    if (state == ST_PROBING) {
      bool eq = true, empty = true;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        uint64_t cur = keys[slot * NW + w];
        eq           = eq && (cur == k[w]);
        empty        = empty && (cur == kEmptyWord);
      }
      if (eq) state = ST_FOUND;
      else if (empty) state = ST_INSERT;
      else if (p == S) state = ST_SPILL;
      else slot = (slot + 1) & smask;
    }
  }
  if (state == ST_PROBING) state = ST_SPILL;
  // insertion rounds: one writer per contended empty slot
  for (int round = 0; round < 33 && __any_sync(kFull, state == ST_INSERT); ++round) {
    const uint32_t im = __ballot_sync(kFull, state == ST_INSERT);
    if (state == ST_INSERT) {
      const uint32_t grp = __match_any_sync(im, slot);
      if ((__ffs(grp) - 1) == lane) {
        // the slot's accumulators are at their identities since init()
#pragma unroll
        for (int w = 0; w < NW; ++w) keys[slot * NW + w] = k[w];
      }
    }
    __syncwarp();
    if (state == ST_INSERT) {
      bool eq = true;
#pragma unroll
      for (int w = 0; w < NW; ++w) eq = eq && (keys[slot * NW + w] == k[w]);
      if (eq) {
        state = ST_FOUND;
      } else {
        state = ST_SPILL;
        for (uint32_t p = 1; p < S; ++p) {
          slot     = (slot + 1) & smask;
          bool e2  = true, em = true;
#pragma unroll
          for (int w = 0; w < NW; ++w) {
            uint64_t cur = keys[slot * NW + w];
            e2           = e2 && (cur == k[w]);
            em           = em && (cur == kEmptyWord);
          }
          if (e2) {
            state = ST_FOUND;
            break;
          }
          if (em) {
            state = ST_INSERT;
            break;
          }
        }
      }
    }
    __syncwarp();
  }
  if (state == ST_INSERT) state = ST_SPILL;
  return state;
}

// Applies the batch's rows to the warp's table.  Lanes on the same slot are
// ranked (__match_any_sync); in round r the lanes of rank r apply their row,
// so every slot has one writer per round and needs no atomics.
template <int NCH>
__device__ __forceinline__ void warp_accumulate(const Plan& plan, unsigned char* tb, const SmemLayout& sl, bool has,
                                                uint32_t slot, const RowVals<NCH>& v, int lane)
{
  const uint32_t m     = __ballot_sync(kFull, has);
  const uint32_t peers = has ? __match_any_sync(m, slot) : 0u;
  const int rank       = __popc(peers & ((1u << lane) - 1u));
  const int rounds     = static_cast<int>(__reduce_max_sync(kFull, has ? static_cast<unsigned>(rank + 1) : 0u));
  for (int rd = 0; rd < rounds; ++rd) {
    if (has && rank == rd) apply_row(plan, tb, sl, slot, v);
    __syncwarp();
  }
}

// ------------------------------------------------------------ finalisation

// Accumulator reads of one slot from a global table or a warp's table.
struct GlobalAccs {
  const TableRef* t;
  __device__ __forceinline__ uint32_t rows(uint64_t s) const { return t->rows[s]; }
  __device__ __forceinline__ uint64_t acc(int a, uint64_t s, int bytes) const
  {
    if (bytes == 4) return reinterpret_cast<const uint32_t*>(t->acc[a])[s];
    return reinterpret_cast<const uint64_t*>(t->acc[a])[s];
  }
};

struct SmemAccs {
  const unsigned char* tb;
  const SmemLayout* sl;
  __device__ __forceinline__ uint32_t rows(uint64_t s) const
  {
    return reinterpret_cast<const uint32_t*>(tb + sl->rows_off)[s];
  }
  __device__ __forceinline__ uint64_t acc(int a, uint64_t s, int bytes) const
  {
    if (bytes == 4) return reinterpret_cast<const uint32_t*>(tb + sl->acc_off[a])[s];
    return reinterpret_cast<const uint64_t*>(tb + sl->acc_off[a])[s];
  }
};

__device__ __forceinline__ void store_bits(void* p, int64_t i, int width, uint64_t v)
{
  switch (width) {
    case 1: reinterpret_cast<uint8_t*>(p)[i] = static_cast<uint8_t>(v); break;
    case 2: reinterpret_cast<uint16_t*>(p)[i] = static_cast<uint16_t>(v); break;
    case 4: reinterpret_cast<uint32_t*>(p)[i] = static_cast<uint32_t>(v); break;
    default: reinterpret_cast<uint64_t*>(p)[i] = v; break;
  }
}

// One group's accumulators of one channel as finalize_from reads them:
// a slot of a table level ...
template <class Accs>
struct SlotView {
  const Accs& A;
  const Channel& ch;
  uint64_t s;
  __device__ __forceinline__ uint32_t rows() const { return A.rows(s); }
  __device__ __forceinline__ uint32_t cnt() const
  {
    return (ch.a_cnt >= 0) ? static_cast<uint32_t>(A.acc(ch.a_cnt, s, 4)) : rows();
  }
  __device__ __forceinline__ uint64_t sum() const { return A.acc(ch.a_sum, s, 8); }
  __device__ __forceinline__ uint64_t sq() const { return A.acc(ch.a_sq, s, 8); }
  __device__ __forceinline__ uint64_t prod() const { return A.acc(ch.a_prod, s, 8); }
  __device__ __forceinline__ uint64_t minmax(bool mn) const
  {
    return A.acc(mn ? ch.a_min : ch.a_max, s, minmax_is64(ch.ptype) ? 8 : 4);
  }
  __device__ __forceinline__ uint64_t shift() const { return A.acc(ch.a_k, s, 8); }
  __device__ __forceinline__ uint64_t s2() const { return A.acc(ch.a_s2, s, 8); }
  __device__ __forceinline__ uint64_t s1() const { return ch.a_s1 >= 0 ? A.acc(ch.a_s1, s, 8) : 0; }
};

// ... or one thread's registers (a group folded by a single lane).  Every
// field holds the same encoding as the table accumulator of that role.
struct ChanAcc {
  uint32_t cnt;   // valid values
  uint64_t mn;    // enc_minmax(., true) of the least value
  uint64_t mx;    // enc_minmax(., false) of the greatest value
  uint64_t sum;   // wrapping integer sum or double bits
  uint64_t sq;    // sum of squares, same encoding as sum
  uint64_t prod;  // product, same encoding as sum
  uint64_t k;     // VAR shift (first non-NaN value) or kShiftUnset
  double s2;      // sum of (x - K)^2
  double s1;      // sum of (x - K) (read for floating channels)
};

struct RegView {
  const ChanAcc& a;
  uint32_t nrows;
  __device__ __forceinline__ uint32_t rows() const { return nrows; }
  __device__ __forceinline__ uint32_t cnt() const { return a.cnt; }
  __device__ __forceinline__ uint64_t sum() const { return a.sum; }
  __device__ __forceinline__ uint64_t sq() const { return a.sq; }
  __device__ __forceinline__ uint64_t prod() const { return a.prod; }
  __device__ __forceinline__ uint64_t minmax(bool mn) const { return mn ? a.mn : a.mx; }
  __device__ __forceinline__ uint64_t shift() const { return a.k; }
  __device__ __forceinline__ uint64_t s2() const { return static_cast<uint64_t>(__double_as_longlong(a.s2)); }
  __device__ __forceinline__ uint64_t s1() const { return static_cast<uint64_t>(__double_as_longlong(a.s1)); }
};

__device__ __forceinline__ void chan_acc_init(ChanAcc& a)
{
  a.cnt  = 0;
  a.mn   = ~0ULL;
  a.mx   = 0;
  a.sum  = 0;
  a.sq   = 0;
  a.prod = 0;
  a.k    = kShiftUnset;
  a.s2   = 0.0;
  a.s1   = 0.0;
}

// The accumulator roles a channel uses, as bits (read once per channel
// instead of once per row).
enum ChanRole : uint32_t { R_MIN = 1, R_MAX = 2, R_SUM = 4, R_SQ = 8, R_PROD = 16, R_VAR = 32 };
__device__ __forceinline__ uint32_t chan_roles(const Channel& ch)
{
  return (ch.a_min >= 0 ? R_MIN : 0u) | (ch.a_max >= 0 ? R_MAX : 0u) | (ch.a_sum >= 0 ? R_SUM : 0u) |
         (ch.a_sq >= 0 ? R_SQ : 0u) | (ch.a_prod >= 0 ? R_PROD : 0u) | (ch.a_k >= 0 ? R_VAR : 0u);
}

// Physical type of a channel: the compile-time PT when it is >= 0 (a
// specialised fold), else the channel's runtime ptype.
template <int PT>
__device__ __forceinline__ int chan_ptype(const Channel& ch)
{
  return PT >= 0 ? PT : ch.ptype;
}
template <int PT>
__device__ __forceinline__ bool chan_is_float(const Channel& ch)
{
  return PT >= 0 ? (PT == P_F32 || PT == P_F64) : ch.is_float != 0;
}

// Folds one valid value (raw bits) into a channel's registers, with the
// arithmetic of apply_row (integers wrap, floats in double, the shift K is
// the first non-NaN value).  Products start from 1 on the first value.
// `roles` is chan_roles(ch).
template <int PT = -1>
__device__ __forceinline__ void chan_acc_add(const Channel& ch, uint32_t roles, ChanAcc& a, uint64_t b)
{
  const int pt     = chan_ptype<PT>(ch);
  const bool first = a.cnt == 0;
  a.cnt += 1;
  if (roles & R_MIN) a.mn = min(a.mn, enc_minmax(b, pt, true));
  if (roles & R_MAX) a.mx = max(a.mx, enc_minmax(b, pt, false));
  double xf;
  if (chan_is_float<PT>(ch)) {
    xf = as_f64(b, pt);
    if (roles & R_SUM) a.sum = static_cast<uint64_t>(__double_as_longlong(__longlong_as_double(static_cast<long long>(a.sum)) + xf));
    if (roles & R_SQ) a.sq = static_cast<uint64_t>(__double_as_longlong(__longlong_as_double(static_cast<long long>(a.sq)) + xf * xf));
    if (roles & R_PROD)
      a.prod = static_cast<uint64_t>(__double_as_longlong(first ? xf : __longlong_as_double(static_cast<long long>(a.prod)) * xf));
  } else {
    const int64_t x = as_i64(b, pt);
    if (roles & R_SUM) a.sum += static_cast<uint64_t>(x);
    if (roles & R_SQ) a.sq += static_cast<uint64_t>(x) * static_cast<uint64_t>(x);
    if (roles & R_PROD) a.prod = first ? static_cast<uint64_t>(x) : a.prod * static_cast<uint64_t>(x);
    xf = (pt == P_U64) ? static_cast<double>(static_cast<uint64_t>(x)) : static_cast<double>(x);
  }
  if (roles & R_VAR) {
    if (a.k == kShiftUnset && !(xf != xf)) a.k = static_cast<uint64_t>(__double_as_longlong(xf));
    const double d = xf - __longlong_as_double(static_cast<long long>(a.k));
    a.s2 += d * d;
    if (chan_is_float<PT>(ch)) a.s1 += d;
  }
}

// Final value and validity of output column `oc` of one group from its
// channel's accumulators (hash_compound_agg_finalizer,
// hash/groupby.cu:183-349); PT as for chan_acc_add.
template <int PT = -1, class View>
__device__ __forceinline__ uint64_t finalize_from(const Channel& ch, const OutCol& oc, const View& V, bool& valid)
{
  const int pt        = chan_ptype<PT>(ch);
  const bool is_float = chan_is_float<PT>(ch);
  const uint32_t rows = V.rows();
  const uint32_t cnt  = V.cnt();
  valid               = cnt > 0;
  uint64_t vbits      = 0;
  switch (oc.kind) {
    case GBX_AGG_COUNT_VALID: vbits = cnt; valid = true; break;
    case GBX_AGG_COUNT_ALL: vbits = rows; valid = true; break;
    case GBX_AGG_SUM:
    case GBX_AGG_SUM_OF_SQUARES:
    case GBX_AGG_PRODUCT: {
      uint64_t raw = (oc.kind == GBX_AGG_SUM) ? V.sum() : (oc.kind == GBX_AGG_PRODUCT ? V.prod() : V.sq());
      if (is_float) {
        double x = __longlong_as_double(static_cast<long long>(raw));
        vbits    = (oc.out_ptype == P_F32) ? __float_as_uint(static_cast<float>(x))
                                           : static_cast<uint64_t>(__double_as_longlong(x));
      } else {
        vbits = raw;  // truncated to the output width on store (wraps like the reference)
      }
      break;
    }
    case GBX_AGG_MIN:
    case GBX_AGG_MAX: {
      bool mn = oc.kind == GBX_AGG_MIN;
      vbits   = dec_minmax(V.minmax(mn), pt, mn);
      break;
    }
    case GBX_AGG_MEAN: {
      if (!valid) break;
      uint64_t raw = V.sum();
      if (oc.out_ptype == P_F64) {
        // integer SUMs are INT64 (target_type): the mean divides the signed sum,
        // as binary_operation(DIV) does on it (hash/groupby.cu:298-304)
        double sum = is_float ? __longlong_as_double(static_cast<long long>(raw))
                              : static_cast<double>(static_cast<int64_t>(raw));
        vbits = static_cast<uint64_t>(__double_as_longlong(sum / static_cast<double>(cnt)));
      } else {
        // duration / decimal MEAN: the SUM wraps to the source width, then
        // integer division of the representation
        int64_t sw = static_cast<int64_t>(raw);
        if (oc.out_width == 4) sw = static_cast<int32_t>(static_cast<uint32_t>(raw));
        vbits = static_cast<uint64_t>(sw / static_cast<int64_t>(cnt));
      }
      break;
    }
    case GBX_AGG_VARIANCE:
    case GBX_AGG_STD:
    case GBX_AGG_M2: {
      int64_t nn = cnt;
      // M2 (group_m2.cu): the centred sum of squares itself, null without values
      const int64_t ddof = oc.kind == GBX_AGG_M2 ? 0 : oc.ddof;
      if (nn == 0 || nn - ddof <= 0) {
        valid = false;
        break;
      }
      uint64_t kb = V.shift();
      double s2   = __longlong_as_double(static_cast<long long>(V.s2()));
      double var;
      if (kb == kShiftUnset) {
        var = s2;  // NaN inputs only
      } else {
        double K  = __longlong_as_double(static_cast<long long>(kb));
        double S1 = shifted_sum(is_float, pt, V.sum(), V.s1(), nn, K);
        double M2 = s2 - S1 * (S1 / static_cast<double>(nn));
        if (M2 < 0.0) M2 = 0.0;
        var = oc.kind == GBX_AGG_M2 ? M2 : M2 / static_cast<double>(nn - ddof);
      }
      if (oc.kind == GBX_AGG_STD) var = sqrt(var);
      vbits = static_cast<uint64_t>(__double_as_longlong(var));
      valid = true;
      break;
    }
    default: break;
  }
  return valid ? vbits : 0;
}

// finalize_from on slot `s` of a table level.
template <class Accs>
__device__ __forceinline__ uint64_t finalize_value(const Plan& plan, const OutCol& oc, const Accs& A, uint64_t s,
                                                   bool& valid)
{
  const Channel& ch = plan.chan[oc.chan];
  return finalize_from(ch, oc, SlotView<Accs>{A, ch, s}, valid);
}

// Decoded key column `c` of a packed key; `valid` false for a null key.
__device__ __forceinline__ uint64_t decode_key(const KeyCol& kc, const uint64_t (&k)[2], bool& valid)
{
  valid = true;
  if (kc.null_bit) valid = ((k[kc.null_word] >> kc.null_shift) & 1ULL) == 0;
  const int bits      = kc.width * 8;
  const uint64_t word = k[kc.word];
  uint64_t v          = (bits == 64) ? word : ((word >> kc.shift) & ((1ULL << bits) - 1));
  return valid ? v : 0;
}

// Or-s a warp's 32 validity bits for rows [base, base + 32) into a bitmask
// whose words the caller zeroed (other warps may own the neighbouring bits).
__device__ __forceinline__ void or_mask_bits(uint32_t* mask, int64_t base, uint32_t bits)
{
  if (bits == 0) return;
  const int64_t w = base >> 5;
  const int sh    = static_cast<int>(base & 31);
  if (sh == 0) {
    atomicOr(mask + w, bits);
  } else {
    const uint32_t lo = bits << sh;
    const uint32_t hi = bits >> (32 - sh);
    if (lo) atomicOr(mask + w, lo);
    if (hi) atomicOr(mask + w + 1, hi);
  }
}

// Null counts of the output columns, indexed like OutPlan::null_counts:
// either straight into the global counters or into per-CTA shared-memory
// counters that the kernel adds to them once at its end (many warps adding
// to the same few global words serialise on them).
struct NullSink {
  unsigned long long* global;
  uint32_t* cta;  // shared memory, or nullptr
  __device__ __forceinline__ void add(int i, uint32_t v) const
  {
    if (cta != nullptr) atomicAdd(cta + i, v);
    else atomicAdd(global + i, static_cast<unsigned long long>(v));
  }
};

constexpr int kNullSlots = kMaxKeyCols + kMaxOut;

// Per-CTA null counters: zeroed before the CTA's first output, flushed by
// every thread of the block after its last (both include __syncthreads).
__device__ __forceinline__ void cta_nulls_zero(uint32_t* c)
{
  for (int i = threadIdx.x; i < kNullSlots; i += blockDim.x) c[i] = 0;
  __syncthreads();
}
__device__ __forceinline__ void cta_nulls_flush(const uint32_t* c, unsigned long long* global)
{
  __syncthreads();
  for (int i = threadIdx.x; i < kNullSlots; i += blockDim.x)
    if (c[i] != 0) atomicAdd(global + i, static_cast<unsigned long long>(c[i]));
}

// Warp-cooperative output of up to 32 groups: lane i writes output row
// base + i from slot `s` when `active` (active lanes form a prefix).  Keys
// are decoded, every result finalised; validity bits are or-ed in one word
// operation per warp and null counts added once per warp.
// The key columns of such a batch of output rows.
__device__ __forceinline__ void warp_write_keys(const Plan& plan, const OutPlan& op, bool active,
                                                const uint64_t (&k)[2], int64_t base, int lane, uint32_t act,
                                                const NullSink& sink)
{
  const int64_t g = base + lane;
  for (int c = 0; c < plan.key.ncols; ++c) {
    const KeyCol& kc = plan.key.cols[c];
    bool valid       = false;
    uint64_t v       = active ? decode_key(kc, k, valid) : 0;
    if (active) store_bits(op.key_data[c], g, kc.width, v);
    if (op.key_mask[c] != nullptr) {
      const uint32_t bits = __ballot_sync(kFull, active && valid);
      if (lane == 0) {
        or_mask_bits(op.key_mask[c], base, bits);
        const uint32_t nulls = __popc(act & ~bits);
        if (nulls) sink.add(c, nulls);
      }
    }
  }
}

template <class Accs>
__device__ __forceinline__ void warp_write_groups(const Plan& plan, const OutPlan& op, const Accs& A, bool active,
                                                  uint64_t s, const uint64_t (&k)[2], int64_t base, int lane,
                                                  uint32_t* cta_nulls = nullptr)
{
  const NullSink sink{op.null_counts, cta_nulls};
  const uint32_t act = __ballot_sync(kFull, active);
  const int64_t g    = base + lane;
  warp_write_keys(plan, op, active, k, base, lane, act, sink);
  for (int o = 0; o < op.nout; ++o) {
    const OutCol& oc = op.out[o];
    bool valid       = false;
    uint64_t v       = active ? finalize_value(plan, oc, A, s, valid) : 0;
    if (active) store_bits(oc.data, g, oc.out_width, v);
    if (oc.mask != nullptr) {
      const uint32_t bits = __ballot_sync(kFull, active && valid);
      if (lane == 0) {
        or_mask_bits(oc.mask, base, bits);
        const uint32_t nulls = __popc(act & ~bits);
        if (nulls) sink.add(kMaxKeyCols + o, nulls);
      }
    }
  }
}

}  // namespace dev
}  // namespace gbx
