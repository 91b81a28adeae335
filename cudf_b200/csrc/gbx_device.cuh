// gbx_device.cuh -- device building blocks of libgbx's hash groupby kernels
// (sm_100a): key packing and hashing, element loads, order-preserving
// encodings, shared/global reductions in explicit state spaces, and the
// bounded open-addressing find-or-insert used by both table levels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gbx_plan.hpp"

namespace gbx {
namespace dev {

// --------------------------------------------------------------- bit access

__device__ __forceinline__ bool bit_valid(const uint32_t* mask, int64_t i)
{
  return mask == nullptr || ((__ldg(mask + (i >> 5)) >> (i & 31)) & 1u);
}

// ---------------------------------------------------------------- hashing

// 64-bit finaliser of MurmurHash3 (Appleby, public domain): a bijective mix.
// The reference hashes rows with MurmurHash3_x86_32 per element folded by
// hash_combine (hashing/detail/murmurhash3_x86_32.cuh:40-130, hashing.hpp:85-88);
// hash values are internal here (group order is unspecified), so the packed
// key is mixed once instead.
__device__ __forceinline__ uint64_t fmix64(uint64_t k)
{
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

template <int NW>
__device__ __forceinline__ uint64_t hash_key(const uint64_t (&k)[NW])
{
  if constexpr (NW == 1) {
    return fmix64(k[0]);
  } else {
    return fmix64(k[0] ^ fmix64(k[1] + 0x9e3779b97f4a7c15ULL));
  }
}

template <int NW>
__device__ __forceinline__ bool key_is_empty(const uint64_t (&k)[NW])
{
  if constexpr (NW == 1) {
    return k[0] == kEmptyWord;
  } else {
    return k[0] == kEmptyWord && k[1] == kEmptyWord;
  }
}

// ------------------------------------------------------------- element loads

__device__ __forceinline__ uint64_t load_bits(const void* p, int64_t i, int width)
{
  switch (width) {
    case 1: return __ldg(reinterpret_cast<const uint8_t*>(p) + i);
    case 2: return __ldg(reinterpret_cast<const uint16_t*>(p) + i);
    case 4: return __ldg(reinterpret_cast<const uint32_t*>(p) + i);
    default: return __ldg(reinterpret_cast<const unsigned long long*>(p) + i);
  }
}

// Buffers of the key columns as a KeyPlan names them.
struct PlanKeyBufs {
  const KeyPlan* kp;
  __device__ __forceinline__ const void* data(int c) const { return kp->cols[c].data; }
  __device__ __forceinline__ const uint32_t* mask(int c) const { return kp->cols[c].mask; }
  __device__ __forceinline__ int64_t offset(int c) const { return kp->cols[c].offset; }
};

// Packs row `row`'s key into NW words, reading column c from bufs.data(c)
// (validity bufs.mask(c), row offset bufs.offset(c)) with the layout of
// kp.cols[c].  Returns false when the row must be skipped (a null key under
// null_policy::EXCLUDE).  Float keys are normalised so that -0.0 == +0.0 and
// every NaN is one key, matching the reference's nan-equal comparator and
// hash normalisation (row_operators.cuh:1285-1312,
// hashing/detail/hash_functions.cuh:41-47).
template <int NW, class Bufs>
__device__ __forceinline__ bool pack_key_from(const KeyPlan& kp, const Bufs& bufs, int64_t row, uint64_t (&k)[NW])
{
#pragma unroll
  for (int w = 0; w < NW; ++w) k[w] = 0;
  for (int c = 0; c < kp.ncols; ++c) {
    const KeyCol& kc = kp.cols[c];
    int64_t i        = row + bufs.offset(c);
    bool valid       = bit_valid(bufs.mask(c), i);
    if (!valid) {
      if (kp.skip_null_rows) return false;
      if (kc.null_bit) {
        k[kc.null_word & (NW - 1)] |= 1ULL << kc.null_shift;
        continue;
      }
    }
    uint64_t v = load_bits(bufs.data(c), i, kc.width);
    if (kc.is_float) {
      if (kc.width == 4) {
        float f = __uint_as_float(static_cast<uint32_t>(v));
        if (f != f) v = 0x7fc00000u;
        else if (f == 0.0f) v = 0;
      } else {
        double d = __longlong_as_double(static_cast<long long>(v));
        if (d != d) v = 0x7ff8000000000000ULL;
        else if (d == 0.0) v = 0;
      }
    } else if (kc.is_bool) {
      v = (v != 0);
    }
    k[kc.word & (NW - 1)] |= v << kc.shift;
  }
  return true;
}

template <int NW>
__device__ __forceinline__ bool pack_key(const KeyPlan& kp, int64_t row, uint64_t (&k)[NW])
{
  return pack_key_from<NW>(kp, PlanKeyBufs{&kp}, row, k);
}

// ------------------------------------------------------------ value loads

__device__ __forceinline__ int64_t dict_index(const Channel& ch, const void* data, int64_t i)
{
  uint64_t b = load_bits(data, i, ch.idx_width);
  if (ch.idx_signed) {
    switch (ch.idx_width) {
      case 1: return static_cast<int8_t>(b);
      case 2: return static_cast<int16_t>(b);
      case 4: return static_cast<int32_t>(b);
      default: return static_cast<int64_t>(b);
    }
  }
  return static_cast<int64_t>(b);
}

// Raw element of a value column with the element layout of `ch` read from
// `data` at row + offset (dictionary resolved through dict_data when it is
// set).  `ok` false on an out-of-range dictionary index (the row is then
// ignored and a status bit set).
__device__ __forceinline__ uint64_t value_bits_at(const Channel& ch, const void* data, int64_t offset,
                                                  const void* dict_data, int64_t dict_offset, int64_t dict_size,
                                                  int64_t row, bool& ok)
{
  const void* base = data;
  int64_t i        = row + offset;
  if (dict_data != nullptr) {
    int64_t k = dict_index(ch, data, i);
    if (k < 0 || k >= dict_size) {
      ok = false;
      return 0;
    }
    base = dict_data;
    i    = k + dict_offset;
  }
  ok = true;
  switch (ch.ptype) {
    case P_I8:
    case P_U8:
    case P_BOOL: return load_bits(base, i, 1);
    case P_I16:
    case P_U16: return load_bits(base, i, 2);
    case P_I32:
    case P_U32:
    case P_F32: return load_bits(base, i, 4);
    default: return load_bits(base, i, 8);
  }
}

__device__ __forceinline__ uint64_t value_bits(const Channel& ch, int64_t row, bool& ok)
{
  return value_bits_at(ch, ch.data, ch.offset, ch.dict_data, ch.dict_offset, ch.dict_size, row, ok);
}

__device__ __forceinline__ int64_t as_i64(uint64_t b, int ptype)
{
  switch (ptype) {
    case P_I8: return static_cast<int8_t>(b);
    case P_I16: return static_cast<int16_t>(b);
    case P_I32: return static_cast<int32_t>(b);
    case P_BOOL: return b != 0;
    default: return static_cast<int64_t>(b);  // I64, U8..U64 (zero-extended)
  }
}

__device__ __forceinline__ double as_f64(uint64_t b, int ptype)
{
  switch (ptype) {
    case P_F32: return static_cast<double>(__uint_as_float(static_cast<uint32_t>(b)));
    case P_F64: return __longlong_as_double(static_cast<long long>(b));
    case P_U64: return static_cast<double>(b);
    default: return static_cast<double>(as_i64(b, ptype));
  }
}

// S1 = sum over a group's valid values of (x - K), K its VAR shift, for the
// centred square sum M2 = sum (x - K)^2 - S1^2 / n.  A floating channel keeps
// S1 as its own accumulator (`s1_raw`, double bits): deriving it from the
// plain sum as sum - n K would cancel and lose every digit of the variance
// once |mean| >> std.  An integer channel's sum is exact (wrapping int64), so
// S1 is the exact wrapping difference sum - n K, read as a signed 64-bit
// value (K is an integer-valued double: the group's first value).
__device__ __forceinline__ double shifted_sum(bool is_float, int ptype, uint64_t sum_raw, uint64_t s1_raw, int64_t n,
                                              double K)
{
  if (is_float) return __longlong_as_double(static_cast<long long>(s1_raw));
  const uint64_t k = ptype == P_U64 ? static_cast<uint64_t>(K) : static_cast<uint64_t>(static_cast<int64_t>(K));
  return static_cast<double>(static_cast<int64_t>(sum_raw - static_cast<uint64_t>(n) * k));
}

// Order-preserving unsigned encodings for MIN/MAX.  NaN maps next to the
// identity so that it loses to every other value and survives only when the
// group's valid values are all NaN (see the oracle's stated NaN order).
__device__ __forceinline__ uint64_t enc_minmax(uint64_t b, int ptype, bool for_min)
{
  switch (ptype) {
    case P_I8: return static_cast<uint32_t>(static_cast<int32_t>(static_cast<int8_t>(b))) ^ 0x80000000u;
    case P_I16: return static_cast<uint32_t>(static_cast<int32_t>(static_cast<int16_t>(b))) ^ 0x80000000u;
    case P_I32: return static_cast<uint32_t>(b) ^ 0x80000000u;
    case P_I64: return b ^ 0x8000000000000000ULL;
    case P_BOOL: return b != 0;
    case P_F32: {
      uint32_t u = static_cast<uint32_t>(b);
      if ((u & 0x7fffffffu) > 0x7f800000u) return for_min ? 0xfffffffeu : 1u;
      return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }
    case P_F64: {
      if ((b & 0x7fffffffffffffffULL) > 0x7ff0000000000000ULL)
        return for_min ? 0xfffffffffffffffeULL : 1ULL;
      return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
    }
    default: return b;  // unsigned
  }
}

__device__ __forceinline__ uint64_t dec_minmax(uint64_t e, int ptype, bool for_min)
{
  switch (ptype) {
    case P_I8:
    case P_I16:
    case P_I32: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(static_cast<uint32_t>(e) ^ 0x80000000u)));
    case P_I64: return e ^ 0x8000000000000000ULL;
    case P_F32: {
      uint32_t u = static_cast<uint32_t>(e);
      if (u == (for_min ? 0xfffffffeu : 1u)) return 0x7fc00000u;
      return (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    }
    case P_F64: {
      if (e == (for_min ? 0xfffffffffffffffeULL : 1ULL)) return 0x7ff8000000000000ULL;
      return (e & 0x8000000000000000ULL) ? (e & 0x7fffffffffffffffULL) : ~e;
    }
    default: return e;
  }
}

__device__ __forceinline__ bool minmax_is64(int ptype)
{
  return ptype == P_I64 || ptype == P_U64 || ptype == P_F64;
}

// -------------------------------------------- reductions in explicit spaces

struct Shared {
  using addr_t = uint32_t;
  static __device__ __forceinline__ void add_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void add_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ void add_f64(addr_t a, double v)
  {
    asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
  }
  static __device__ __forceinline__ void min_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.shared.min.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void max_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.shared.max.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void min_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.shared.min.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ void max_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ uint64_t cas_u64(addr_t a, uint64_t c, uint64_t v)
  {
    uint64_t o;
    asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;" : "=l"(o) : "r"(a), "l"(c), "l"(v) : "memory");
    return o;
  }
  static __device__ __forceinline__ uint32_t cas_u32(addr_t a, uint32_t c, uint32_t v)
  {
    uint32_t o;
    asm volatile("atom.shared.cas.b32 %0, [%1], %2, %3;" : "=r"(o) : "r"(a), "r"(c), "r"(v) : "memory");
    return o;
  }
  static __device__ __forceinline__ uint64_t ld_u64(addr_t a)
  {
    uint64_t v;
    asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
    return v;
  }
  static __device__ __forceinline__ uint32_t ld_u32(addr_t a)
  {
    uint32_t v;
    asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
  }
  static __device__ __forceinline__ void cas128(addr_t a, uint64_t c0, uint64_t c1, uint64_t v0,
                                                uint64_t v1, uint64_t& o0, uint64_t& o1)
  {
    asm volatile(
      "{\n\t.reg .b128 c, v, o;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 v, {%4, %5};\n\t"
      "atom.shared.cas.b128 o, [%6], c, v;\n\t"
      "mov.b128 {%0, %1}, o;\n\t}"
      : "=l"(o0), "=l"(o1)
      : "l"(c0), "l"(c1), "l"(v0), "l"(v1), "r"(a)
      : "memory");
  }
};

struct Global {
  using addr_t = uint64_t;
  static __device__ __forceinline__ void add_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void add_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ void add_f64(addr_t a, double v)
  {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(a), "d"(v) : "memory");
  }
  static __device__ __forceinline__ void min_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.global.min.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void max_u32(addr_t a, uint32_t v)
  {
    asm volatile("red.global.max.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
  }
  static __device__ __forceinline__ void min_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.global.min.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ void max_u64(addr_t a, uint64_t v)
  {
    asm volatile("red.global.max.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
  }
  static __device__ __forceinline__ uint64_t cas_u64(addr_t a, uint64_t c, uint64_t v)
  {
    uint64_t o;
    asm volatile("atom.global.cas.b64 %0, [%1], %2, %3;" : "=l"(o) : "l"(a), "l"(c), "l"(v) : "memory");
    return o;
  }
  static __device__ __forceinline__ uint32_t cas_u32(addr_t a, uint32_t c, uint32_t v)
  {
    uint32_t o;
    asm volatile("atom.global.cas.b32 %0, [%1], %2, %3;" : "=r"(o) : "l"(a), "r"(c), "r"(v) : "memory");
    return o;
  }
  static __device__ __forceinline__ uint64_t ld_u64(addr_t a)
  {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
    return v;
  }
  static __device__ __forceinline__ uint32_t ld_u32(addr_t a)
  {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
    return v;
  }
  static __device__ __forceinline__ void cas128(addr_t a, uint64_t c0, uint64_t c1, uint64_t v0,
                                                uint64_t v1, uint64_t& o0, uint64_t& o1)
  {
    asm volatile(
      "{\n\t.reg .b128 c, v, o;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 v, {%4, %5};\n\t"
      "atom.global.cas.b128 o, [%6], c, v;\n\t"
      "mov.b128 {%0, %1}, o;\n\t}"
      : "=l"(o0), "=l"(o1)
      : "l"(c0), "l"(c1), "l"(v0), "l"(v1), "l"(a)
      : "memory");
  }
};

// -------------------------------------------------------- find-or-insert

// Linear probing over `mask + 1` slots starting at the hash's home slot.
// Keys are stored as NW consecutive words per slot.  Returns the slot holding
// `k` (inserting it into an empty slot if absent) or -1 when `max_probes`
// slots were examined without success.  Every loop is bounded.
template <class Space, int NW>
__device__ __forceinline__ int64_t find_or_insert(typename Space::addr_t keys,
                                                  uint64_t mask,
                                                  const uint64_t (&k)[NW],
                                                  uint64_t h,
                                                  uint32_t max_probes)
{
  uint64_t s = h & mask;
  for (uint32_t p = 0; p < max_probes; ++p) {
    typename Space::addr_t a = keys + static_cast<typename Space::addr_t>(s * NW * 8);
    if constexpr (NW == 1) {
      uint64_t cur = Space::ld_u64(a);
      if (cur == k[0]) return static_cast<int64_t>(s);
      if (cur == kEmptyWord) {
        uint64_t old = Space::cas_u64(a, kEmptyWord, k[0]);
        if (old == kEmptyWord || old == k[0]) return static_cast<int64_t>(s);
      }
    } else {
      uint64_t c0 = Space::ld_u64(a);
      uint64_t c1 = Space::ld_u64(a + 8);
      if (c0 == k[0] && c1 == k[1]) return static_cast<int64_t>(s);
      if (c0 == kEmptyWord || c1 == kEmptyWord) {
        // empty or being written: the 128-bit CAS decides
        uint64_t o0, o1;
        Space::cas128(a, kEmptyWord, kEmptyWord, k[0], k[1], o0, o1);
        if ((o0 == kEmptyWord && o1 == kEmptyWord) || (o0 == k[0] && o1 == k[1]))
          return static_cast<int64_t>(s);
      }
    }
    s = (s + 1) & mask;
  }
  return -1;
}

// Lanes of the warp (among `act`) whose digit of `width` (<= 8) bits equals
// this lane's: one ballot per digit bit.  The same lane sets as a match on
// the digit, on the ALU instead of the pipe that serialises matches.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, int width, uint32_t act)
{
  uint32_t peers = act;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    if (b >= width) break;
    const uint32_t v = __ballot_sync(0xffffffffu, (d >> b) & 1u);
    peers &= ((d >> b) & 1u) ? v : ~v;
  }
  return peers;
}

}  // namespace dev
}  // namespace gbx
