// gbx_table.cuh -- table-level device operations shared by libgbx's
// aggregation kernels: identities, per-row accumulation into a table level
// (shared or global memory), merging a partial slot into the global table,
// and the global find-or-insert with its reserved all-ones slot.
#pragma once

#include "gbx_device.cuh"
#include "gbx_kernels.hpp"

namespace gbx {
namespace dev {

// ------------------------------------------------------------ identities

__device__ __forceinline__ uint64_t identity_bits(int kind)
{
  switch (kind) {
    case A_U32_MIN: return 0xffffffffULL;
    case A_U64_MIN: return 0xffffffffffffffffULL;
    case A_F64_SHIFT: return kShiftUnset;
    case A_I64_MUL: return 1ULL;
    case A_F64_MUL: return 0x3ff0000000000000ULL;  // 1.0
    case A_U64_ARGMIN: return 0xffffffffffffffffULL;
    case A_I32_ARGMIN_CAS:
    case A_I32_ARGMAX_CAS: return 0xffffffffULL;  // -1 sentinel
    default: return 0;  // adds, max encodings
  }
}

// ---------------------------------------------------- per-row accumulation

// Addressing of one table level: base address (in the state space of
// `Space`) of the row counts and of each accumulator array.  Holds a pointer
// to the descriptor, which kernels take as a __grid_constant__ parameter, so
// runtime-indexed reads come from parameter space instead of a local copy.
template <class Space>
struct Level;

template <>
struct Level<Global> {
  const TableRef* t;
  __device__ __forceinline__ uint64_t rows() const { return reinterpret_cast<uint64_t>(t->rows); }
  __device__ __forceinline__ uint64_t acc(int a) const { return reinterpret_cast<uint64_t>(t->acc[a]); }
};

template <>
struct Level<Shared> {
  uint32_t base;  // shared-memory address of the table
  const SmemLayout* sl;
  __device__ __forceinline__ uint32_t rows() const { return base + sl->rows_off; }
  __device__ __forceinline__ uint32_t acc(int a) const { return base + sl->acc_off[a]; }
};

template <class Space>
__device__ __forceinline__ void mul_cas_i64(typename Space::addr_t a, int64_t x, int32_t* status)
{
  uint64_t cur = Space::ld_u64(a);
  for (int it = 0; it < (1 << 20); ++it) {
    uint64_t nv  = static_cast<uint64_t>(static_cast<int64_t>(cur) * x);
    uint64_t old = Space::cas_u64(a, cur, nv);
    if (old == cur) return;
    cur = old;
  }
  atomicOr(status, S_SPIN_LIMIT);
}

template <class Space>
__device__ __forceinline__ void mul_cas_f64(typename Space::addr_t a, double x, int32_t* status)
{
  uint64_t cur = Space::ld_u64(a);
  for (int it = 0; it < (1 << 20); ++it) {
    double nvd   = __longlong_as_double(static_cast<long long>(cur)) * x;
    uint64_t nv  = static_cast<uint64_t>(__double_as_longlong(nvd));
    uint64_t old = Space::cas_u64(a, cur, nv);
    if (old == cur) return;
    cur = old;
  }
  atomicOr(status, S_SPIN_LIMIT);
}

// Shift of a VAR accumulator: the recorded K, recording `x` first if unset.
template <class Space>
__device__ __forceinline__ double get_shift(typename Space::addr_t a, double x)
{
  uint64_t kb = Space::ld_u64(a);
  if (kb == kShiftUnset && !(x != x)) {
    uint64_t xb  = static_cast<uint64_t>(__double_as_longlong(x));
    uint64_t old = Space::cas_u64(a, kShiftUnset, xb);
    kb           = (old == kShiftUnset) ? xb : old;
  }
  return __longlong_as_double(static_cast<long long>(kb));
}

// ------------------------------------------------------------ ARGMIN / ARGMAX

// Order key of a value for ARGMIN (`for_min`) or ARGMAX: the MIN/MAX encoding
// (NaN loses to every number) with -0.0 folded into +0.0, so that the two
// zeros tie as they do under the reference's `<` / `>` comparisons
// (detail/aggregation/aggregation.cuh:436-491).  Ties go to the lowest row.
__device__ __forceinline__ uint64_t arg_order(uint64_t b, int ptype, bool for_min)
{
  if (ptype == P_F32 && (static_cast<uint32_t>(b) << 1) == 0) b = 0;
  if (ptype == P_F64 && (b << 1) == 0) b = 0;
  return enc_minmax(b, ptype, for_min);
}

// Values of at most 32 bits: one 64-bit word per group, the order key in the
// high half and the row (ARGMIN) or its complement (ARGMAX) in the low half,
// so that a single 64-bit min / max keeps the extreme value and, among equal
// values, the lowest row.  Rows are below 2^31, so neither identity (all
// ones for ARGMIN, zero for ARGMAX) is a packed row.
__device__ __forceinline__ uint64_t arg_pack(uint64_t order, bool for_min, uint32_t row)
{
  return (order << 32) | (for_min ? row : ~row);
}

// 64-bit values: the group's row index, replaced by compare-and-swap while
// the new row's value beats the value re-read at the stored row (the
// reference's loop, aggregation.cuh:449-458, with the lowest-row tie rule).
// Values never change during a call, so the loop ends with the best row.
template <class Space>
__device__ __forceinline__ void arg_cas(typename Space::addr_t a, const Channel& ch, uint64_t order, uint32_t row,
                                     bool for_min, int32_t* status)
{
  uint32_t cur = Space::ld_u32(a);
  for (int it = 0; it < (1 << 20); ++it) {
    if (cur != 0xffffffffu) {
      bool ok;
      const uint64_t held = arg_order(value_bits(ch, cur, ok), ch.ptype, for_min);
      const bool wins     = for_min ? order < held : order > held;
      if (!wins && !(order == held && row < cur)) return;
    }
    const uint32_t old = Space::cas_u32(a, cur, row);
    if (old == cur) return;
    cur = old;
  }
  atomicOr(status, S_SPIN_LIMIT);
}

// Folds (value bits `b`, row) into a channel's ARGMIN / ARGMAX accumulator at
// `acc` (the array base) for slot `slot`.
template <class Space>
__device__ __forceinline__ void arg_update(typename Space::addr_t acc, int64_t slot, const Channel& ch, uint64_t b,
                                        uint32_t row, bool for_min, int32_t* status)
{
  using A              = typename Space::addr_t;
  const uint64_t order = arg_order(b, ch.ptype, for_min);
  if (minmax_is64(ch.ptype)) {
    arg_cas<Space>(acc + static_cast<A>(slot * 4), ch, order, row, for_min, status);
  } else if (for_min) {
    Space::min_u64(acc + static_cast<A>(slot * 8), arg_pack(order, true, row));
  } else {
    Space::max_u64(acc + static_cast<A>(slot * 8), arg_pack(order, false, row));
  }
}

// Merges a partial table's ARGMIN / ARGMAX accumulator (slot `s` at `src`)
// into the global one (slot `g` at `dst`).
template <class Src>
__device__ __forceinline__ void arg_merge(typename Src::addr_t src, int64_t s, uint64_t dst, int64_t g,
                                       const Channel& ch, bool for_min, int32_t* status)
{
  using SA = typename Src::addr_t;
  if (minmax_is64(ch.ptype)) {
    const uint32_t row = Src::ld_u32(src + static_cast<SA>(s * 4));
    if (row == 0xffffffffu) return;
    bool ok;
    const uint64_t order = arg_order(value_bits(ch, row, ok), ch.ptype, for_min);
    arg_cas<Global>(dst + static_cast<uint64_t>(g * 4), ch, order, row, for_min, status);
  } else {
    const uint64_t w = Src::ld_u64(src + static_cast<SA>(s * 8));
    if (for_min) Global::min_u64(dst + static_cast<uint64_t>(g * 8), w);
    else Global::max_u64(dst + static_cast<uint64_t>(g * 8), w);
  }
}

// ------------------------------------------------------------- row sources

// Rows of the caller's columns as the plan names them.
struct RowSource {
  const Plan* plan;
  template <int NW>
  __device__ __forceinline__ bool key(int64_t r, uint64_t (&k)[NW]) const
  {
    return pack_key<NW>(plan->key, r, k);
  }
  // Raw bits of channel c at row r; false for a null value (or an
  // out-of-range dictionary index, which also sets S_BAD_INDEX).
  __device__ __forceinline__ bool value(int c, int64_t r, uint64_t& b, int32_t* status) const
  {
    const Channel& ch = plan->chan[c];
    if (!bit_valid(ch.mask, r + ch.offset)) return false;
    bool ok;
    b = value_bits(ch, r, ok);
    if (!ok) {
      atomicOr(status, S_BAD_INDEX);
      return false;
    }
    return true;
  }
};

// Folds row `row` of `src` into slot `slot` of a table level (aggregate_row,
// detail/aggregation/aggregation.cuh:558-573, with update_target_element's
// null skipping, :116-491).  ARGMIN / ARGMAX accumulators are updated only in
// the `kArg` instantiations (kernels launched for plans that carry them), so
// the other kernels keep their registers.
template <class Space, class Src, bool kArg = false>
__device__ __forceinline__ void accumulate_row_from(const Plan& plan,
                                                    const Src& src,
                                                    const Level<Space>& L,
                                                    int64_t slot,
                                                    int64_t row,
                                                    int32_t* status)
{
  using A = typename Space::addr_t;
  Space::add_u32(L.rows() + static_cast<A>(slot * 4), 1u);
  for (int c = 0; c < plan.nchan; ++c) {
    const Channel& ch = plan.chan[c];
    uint64_t b;
    if (!src.value(c, row, b, status)) continue;
    if (ch.a_cnt >= 0) Space::add_u32(L.acc(ch.a_cnt) + static_cast<A>(slot * 4), 1u);
    const bool is64 = minmax_is64(ch.ptype);
    if (ch.a_min >= 0) {
      uint64_t e = enc_minmax(b, ch.ptype, true);
      if (is64) Space::min_u64(L.acc(ch.a_min) + static_cast<A>(slot * 8), e);
      else Space::min_u32(L.acc(ch.a_min) + static_cast<A>(slot * 4), static_cast<uint32_t>(e));
    }
    if (ch.a_max >= 0) {
      uint64_t e = enc_minmax(b, ch.ptype, false);
      if (is64) Space::max_u64(L.acc(ch.a_max) + static_cast<A>(slot * 8), e);
      else Space::max_u32(L.acc(ch.a_max) + static_cast<A>(slot * 4), static_cast<uint32_t>(e));
    }
    if constexpr (kArg) {
      if (ch.a_amin >= 0) arg_update<Space>(L.acc(ch.a_amin), slot, ch, b, static_cast<uint32_t>(row), true, status);
      if (ch.a_amax >= 0) arg_update<Space>(L.acc(ch.a_amax), slot, ch, b, static_cast<uint32_t>(row), false, status);
    }
    if (ch.is_float) {
      double x = as_f64(b, ch.ptype);
      if (ch.a_sum >= 0) Space::add_f64(L.acc(ch.a_sum) + static_cast<A>(slot * 8), x);
      if (ch.a_sq >= 0) Space::add_f64(L.acc(ch.a_sq) + static_cast<A>(slot * 8), x * x);
      if (ch.a_prod >= 0) mul_cas_f64<Space>(L.acc(ch.a_prod) + static_cast<A>(slot * 8), x, status);
      if (ch.a_k >= 0) {
        double K = get_shift<Space>(L.acc(ch.a_k) + static_cast<A>(slot * 8), x);
        double d = x - K;
        Space::add_f64(L.acc(ch.a_s2) + static_cast<A>(slot * 8), d * d);
        Space::add_f64(L.acc(ch.a_s1) + static_cast<A>(slot * 8), d);
      }
    } else {
      int64_t x = as_i64(b, ch.ptype);
      if (ch.a_sum >= 0) Space::add_u64(L.acc(ch.a_sum) + static_cast<A>(slot * 8), static_cast<uint64_t>(x));
      if (ch.a_sq >= 0)
        Space::add_u64(L.acc(ch.a_sq) + static_cast<A>(slot * 8),
                       static_cast<uint64_t>(x) * static_cast<uint64_t>(x));
      if (ch.a_prod >= 0) mul_cas_i64<Space>(L.acc(ch.a_prod) + static_cast<A>(slot * 8), x, status);
      if (ch.a_k >= 0) {
        double xf = (ch.ptype == P_U64) ? static_cast<double>(static_cast<uint64_t>(x))
                                        : static_cast<double>(x);
        double K = get_shift<Space>(L.acc(ch.a_k) + static_cast<A>(slot * 8), xf);
        double d = xf - K;
        Space::add_f64(L.acc(ch.a_s2) + static_cast<A>(slot * 8), d * d);
      }
    }
  }
}

template <class Space, bool kArg = false>
__device__ __forceinline__ void accumulate_row(const Plan& plan,
                                               const Level<Space>& L,
                                               int64_t slot,
                                               int64_t row,
                                               int32_t* status)
{
  accumulate_row_from<Space, RowSource, kArg>(plan, RowSource{&plan}, L, slot, row, status);
}

// Merges slot `s` of a (shared-memory) partial level into slot `g` of the
// global level (ARGMIN / ARGMAX in the `kArg` instantiations only).
template <class Src, bool kArg = false>
__device__ __forceinline__ void merge_slot(const Plan& plan,
                                           const Level<Src>& S,
                                           int64_t s,
                                           const Level<Global>& G,
                                           int64_t g,
                                           int32_t* status)
{
  using SA           = typename Src::addr_t;
  uint32_t rows      = Src::ld_u32(S.rows() + static_cast<SA>(s * 4));
  Global::add_u32(G.rows() + static_cast<uint64_t>(g * 4), rows);
  for (int c = 0; c < plan.nchan; ++c) {
    const Channel& ch = plan.chan[c];
    uint32_t n        = rows;
    if (ch.a_cnt >= 0) {
      n = Src::ld_u32(S.acc(ch.a_cnt) + static_cast<SA>(s * 4));
      Global::add_u32(G.acc(ch.a_cnt) + static_cast<uint64_t>(g * 4), n);
    }
    if (n == 0) continue;
    const bool is64 = minmax_is64(ch.ptype);
    if (ch.a_min >= 0) {
      if (is64) Global::min_u64(G.acc(ch.a_min) + static_cast<uint64_t>(g * 8), Src::ld_u64(S.acc(ch.a_min) + static_cast<SA>(s * 8)));
      else Global::min_u32(G.acc(ch.a_min) + static_cast<uint64_t>(g * 4), Src::ld_u32(S.acc(ch.a_min) + static_cast<SA>(s * 4)));
    }
    if (ch.a_max >= 0) {
      if (is64) Global::max_u64(G.acc(ch.a_max) + static_cast<uint64_t>(g * 8), Src::ld_u64(S.acc(ch.a_max) + static_cast<SA>(s * 8)));
      else Global::max_u32(G.acc(ch.a_max) + static_cast<uint64_t>(g * 4), Src::ld_u32(S.acc(ch.a_max) + static_cast<SA>(s * 4)));
    }
    if constexpr (kArg) {
      if (ch.a_amin >= 0) arg_merge<Src>(S.acc(ch.a_amin), s, G.acc(ch.a_amin), g, ch, true, status);
      if (ch.a_amax >= 0) arg_merge<Src>(S.acc(ch.a_amax), s, G.acc(ch.a_amax), g, ch, false, status);
    }
    if (ch.is_float) {
      if (ch.a_sum >= 0)
        Global::add_f64(G.acc(ch.a_sum) + static_cast<uint64_t>(g * 8),
                        __longlong_as_double(static_cast<long long>(Src::ld_u64(S.acc(ch.a_sum) + static_cast<SA>(s * 8)))));
      if (ch.a_sq >= 0)
        Global::add_f64(G.acc(ch.a_sq) + static_cast<uint64_t>(g * 8),
                        __longlong_as_double(static_cast<long long>(Src::ld_u64(S.acc(ch.a_sq) + static_cast<SA>(s * 8)))));
      if (ch.a_prod >= 0)
        mul_cas_f64<Global>(G.acc(ch.a_prod) + static_cast<uint64_t>(g * 8),
                            __longlong_as_double(static_cast<long long>(Src::ld_u64(S.acc(ch.a_prod) + static_cast<SA>(s * 8)))),
                            status);
    } else {
      if (ch.a_sum >= 0)
        Global::add_u64(G.acc(ch.a_sum) + static_cast<uint64_t>(g * 8), Src::ld_u64(S.acc(ch.a_sum) + static_cast<SA>(s * 8)));
      if (ch.a_sq >= 0)
        Global::add_u64(G.acc(ch.a_sq) + static_cast<uint64_t>(g * 8), Src::ld_u64(S.acc(ch.a_sq) + static_cast<SA>(s * 8)));
      if (ch.a_prod >= 0)
        mul_cas_i64<Global>(G.acc(ch.a_prod) + static_cast<uint64_t>(g * 8),
                            static_cast<int64_t>(Src::ld_u64(S.acc(ch.a_prod) + static_cast<SA>(s * 8))), status);
    }
    if (ch.a_k >= 0) {
      uint64_t kpb = Src::ld_u64(S.acc(ch.a_k) + static_cast<SA>(s * 8));
      double s2p   = __longlong_as_double(static_cast<long long>(Src::ld_u64(S.acc(ch.a_s2) + static_cast<SA>(s * 8))));
      const uint64_t s1b = ch.a_s1 >= 0 ? Src::ld_u64(S.acc(ch.a_s1) + static_cast<SA>(s * 8)) : 0;
      if (kpb == kShiftUnset) {
        // every valid value was NaN: the partial sums are NaN already
        Global::add_f64(G.acc(ch.a_s2) + static_cast<uint64_t>(g * 8), s2p);
        if (ch.a_s1 >= 0) Global::add_f64(G.acc(ch.a_s1) + static_cast<uint64_t>(g * 8), __longlong_as_double(static_cast<long long>(s1b)));
      } else {
        // re-centre the partial sums on the global shift: with d = Kp - Kg,
        // sum (x-Kg)^2 = sum (x-Kp)^2 + 2 d S1 + n d^2, sum (x-Kg) = S1 + n d
        double Kp = __longlong_as_double(static_cast<long long>(kpb));
        double Kg = get_shift<Global>(G.acc(ch.a_k) + static_cast<uint64_t>(g * 8), Kp);
        double S1 = shifted_sum(ch.is_float, ch.ptype, Src::ld_u64(S.acc(ch.a_sum) + static_cast<SA>(s * 8)), s1b, n, Kp);
        double d  = Kp - Kg;
        Global::add_f64(G.acc(ch.a_s2) + static_cast<uint64_t>(g * 8), s2p + 2.0 * d * S1 + static_cast<double>(n) * d * d);
        if (ch.a_s1 >= 0) Global::add_f64(G.acc(ch.a_s1) + static_cast<uint64_t>(g * 8), S1 + static_cast<double>(n) * d);
      }
    }
  }
}

__device__ __forceinline__ Level<Global> global_level(const TableRef& t) { return Level<Global>{&t}; }

// Global find-or-insert for one key, including the reserved all-ones slot.
template <int NW>
__device__ __forceinline__ int64_t global_slot(const TableRef& t,
                                               const uint64_t (&k)[NW],
                                               uint32_t max_probes)
{
  if (key_is_empty<NW>(k)) {
    if (Global::ld_u32(reinterpret_cast<uint64_t>(t.special_used)) == 0) atomicExch(t.special_used, 1u);
    return static_cast<int64_t>(t.cap);
  }
  int64_t s = find_or_insert<Global, NW>(reinterpret_cast<uint64_t>(t.keys), t.cap - 1, k, hash_key<NW>(k),
                                         max_probes);
  if (s < 0) atomicOr(t.status, S_TABLE_FULL);
  return s;
}

}  // namespace dev
}  // namespace gbx
