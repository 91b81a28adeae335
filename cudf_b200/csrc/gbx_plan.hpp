// gbx_plan.hpp -- plan descriptors shared by the host orchestration and the
// sm_100a kernels of libgbx (hash groupby-aggregation).
//
// A groupby call is lowered to:
//   * a KeyPlan: how each key column's bits are packed into one or two 64-bit
//     table words (fixed-width and dictionary keys, optional null bit per
//     column under null_policy::INCLUDE; rows with a null key are skipped under
//     EXCLUDE, as bitmask_and + the row filter do in the reference,
//     cpp/src/groupby/hash/groupby.cu:482-485 and groupby_kernels.cuh:98-105);
//   * one Channel per distinct value column, naming the accumulators it needs
//     (the reference flattens MEAN/VAR/STD into SUM + COUNT_VALID,
//     hash/groupby.cu:113-181, 351-383; here VAR adds a shift and a shifted
//     sum of squares so it needs no second pass over the rows);
//   * a TableRef: the open-addressing table (keys + one array per accumulator,
//     slot-major SoA) in global memory, and the same layout in shared memory
//     for the per-CTA privatised tables.
#pragma once

#include <stdint.h>

namespace gbx {

constexpr int kMaxKeyCols  = 8;
constexpr int kMaxChannels = 8;
constexpr int kMaxAccs     = 48;

// Physical element codes (after dictionary resolution).
enum PhysType : int8_t {
  P_I8 = 0,
  P_I16,
  P_I32,
  P_I64,
  P_U8,
  P_U16,
  P_U32,
  P_U64,
  P_F32,
  P_F64,
  P_BOOL,
  P_NONE
};

// Bytes of one element of a physical type.
constexpr int pt_width(int pt)
{
  return (pt == P_I8 || pt == P_U8 || pt == P_BOOL) ? 1 : (pt == P_I16 || pt == P_U16) ? 2
         : (pt == P_I32 || pt == P_U32 || pt == P_F32)                                 ? 4
                                                                                        : 8;
}

// Accumulator element kinds: decide identity, merge op and width.
enum AccKind : int8_t {
  A_U32_ADD = 0,  // counts
  A_I64_ADD,      // integer SUM / SUM_OF_SQUARES (wrapping, like atomicAdd on u64)
  A_F64_ADD,      // floating SUM / SUM_OF_SQUARES / shifted square sums
  A_U32_MIN,      // order-preserving encoding of <=32-bit values
  A_U32_MAX,
  A_U64_MIN,      // order-preserving encoding of 64-bit values
  A_U64_MAX,
  A_F64_SHIFT,    // VAR shift K: first non-NaN value seen (sentinel until set)
  A_I64_MUL,      // integer PRODUCT
  A_F64_MUL,      // floating PRODUCT
  A_U64_ARGMIN,   // (encoded value << 32 | row) for <=32-bit values
  A_U64_ARGMAX,   // (encoded value << 32 | ~row) for <=32-bit values
  A_I32_ARGMIN_CAS,  // row index, CAS loop comparing re-read values (64-bit values)
  A_I32_ARGMAX_CAS
};

__host__ __device__ inline int acc_bytes(int kind)
{
  return (kind == A_U32_ADD || kind == A_U32_MIN || kind == A_U32_MAX ||
          kind == A_I32_ARGMIN_CAS || kind == A_I32_ARGMAX_CAS)
           ? 4
           : 8;
}

// Bit pattern of the VAR shift before a value has been recorded (a signalling
// NaN payload that no arithmetic produces; NaN inputs never become a shift).
constexpr uint64_t kShiftUnset = 0x7ff4000000000001ULL;
constexpr uint64_t kEmptyWord  = 0xffffffffffffffffULL;

struct KeyCol {
  const void* data;       // element 0 of the buffer (offset applied by `offset`)
  const uint32_t* mask;   // validity (nullptr: all valid)
  int64_t offset;
  int8_t width;           // bytes: 1, 2, 4, 8
  int8_t is_float;        // normalise -0.0 / NaN
  int8_t is_bool;         // normalise to 0/1
  int8_t null_bit;        // 1: a null bit is packed (INCLUDE policy, column has a mask)
  int8_t word;            // table word (0 or 1) holding this column
  int8_t shift;           // bit offset of the value inside the word
  int8_t null_shift;      // bit offset of the null bit
  int8_t is_signed;       // for decoding (sign of the key type)
  int8_t null_word;       // table word holding the null bit
  int8_t pad[7];
};

struct KeyPlan {
  int32_t ncols;
  int32_t nwords;         // 1 or 2
  int32_t skip_null_rows; // EXCLUDE and some key column has a mask
  int32_t bits_used;      // total packed bits (< 64*nwords => the empty key cannot occur)
  KeyCol cols[kMaxKeyCols];
};

// Accumulator needs of a channel.
enum ChanNeed : uint32_t {
  N_CNT  = 1u << 0,
  N_SUM  = 1u << 1,
  N_MIN  = 1u << 2,
  N_MAX  = 1u << 3,
  N_SQ   = 1u << 4,
  N_VAR  = 1u << 5,
  N_PROD = 1u << 6,
  N_AMIN = 1u << 7,
  N_AMAX = 1u << 8
};

struct Channel {
  const void* data;         // values (or dictionary indices)
  const uint32_t* mask;     // validity of the column (nullptr: all valid)
  int64_t offset;
  const void* dict_data;    // dictionary keys (nullptr: not a dictionary column)
  int64_t dict_offset;
  int64_t dict_size;        // number of dictionary keys (index bound)
  int8_t ptype;             // PhysType of the value (dictionary keys' type)
  int8_t idx_width;         // dictionary index width in bytes
  int8_t idx_signed;
  int8_t is_float;          // ptype is F32/F64
  uint32_t need;            // ChanNeed bits
  // accumulator indices into TableRef::acc (-1: absent); a_s1 (floating
  // channels with VAR/STD only) is the shifted sum sum(x - K)
  int8_t a_cnt, a_sum, a_min, a_max, a_sq, a_k, a_s2, a_prod, a_amin, a_amax, a_s1;
  int8_t pad[1];
};

struct TableRef {
  uint64_t* keys;           // (cap + 1) * nwords words; slot `cap` is the reserved slot
  uint32_t* rows;           // per-slot row count (COUNT_ALL)
  uint32_t* special_used;   // 1 when the reserved slot holds the all-ones key
  void* acc[kMaxAccs];
  uint64_t cap;             // power of two
  int32_t* status;          // device status word
};

struct AccLayout {
  int32_t nacc;
  int8_t kind[kMaxAccs];
};

struct Plan {
  KeyPlan key;
  int32_t nchan;
  Channel chan[kMaxChannels];
  AccLayout acc;
};

// True when some channel of the plan carries an ARGMIN or ARGMAX accumulator.
inline bool plan_has_arg(const Plan& plan)
{
  for (int c = 0; c < plan.nchan; ++c)
    if (plan.chan[c].a_amin >= 0 || plan.chan[c].a_amax >= 0) return true;
  return false;
}

// Device status bits.
enum StatusBits : int32_t {
  S_TABLE_FULL   = 1,  // a global probe sequence hit its limit: retry with a larger table
  S_SPIN_LIMIT   = 2,  // a bounded CAS / publication loop gave up
  S_BAD_INDEX    = 4,  // a dictionary index was out of range
  S_CHECK_FAILED = 8   // a consistency check of the partitioned path failed (rows out of bucket order)
};

}  // namespace gbx
