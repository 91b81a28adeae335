// gbx_kernels.cu -- sm_100a kernels of libgbx's hash groupby-aggregation.
//
// Replaces the reference's per-row thrust::for_each_n over a cuco::static_set
// of row indices with row-count-sized "sparse" result columns
// (cpp/src/groupby/hash/groupby.cu:424-504, groupby_kernels.cuh:98-105) by:
//   * k_sample_distinct  -- a sampled distinct count that sizes the tables;
//   * k_init_table       -- identity fill of a capacity-sized global table
//                           (K2 of the reference writes N-row columns instead);
//   * k_agg_privatized   -- per-CTA shared-memory tables with inline packed
//                           keys, spilling to the global table when full and
//                           flushed into it at the end (K1+K3 fused);
//   * k_agg_global       -- every row updates the global table directly;
//   * k_finalize         -- dense outputs: keys decoded from the packed key,
//                           SUM/COUNT/MIN/MAX/MEAN/VAR/STD finalised and
//                           validity bitmasks written by warp ballots
//                           (K4/K6/K7/K8/K9 fused).
// VAR/STD need no second pass over the rows (the reference's K5,
// multi_pass_kernels.cuh:35-112): each group keeps a shift K (its first
// non-NaN value) and the sum of (x - K)^2; partial tables are merged with the
// shifted-sums identity sum((x-K2)^2) = sum((x-K1)^2) + 2 d S1 + n d^2,
// d = K1 - K2, S1 = sum(x) - n K1 (Chan, Golub & LeVeque, 1983).
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "gbx_kernels.hpp"
#include "gbx_table.cuh"

namespace gbx {

using namespace dev;

// ----------------------------------------------------------------- kernels

__global__ void k_init_table(const __grid_constant__ TableRef t, const __grid_constant__ AccLayout al, int nwords)
{
  const uint64_t n      = t.cap + 1;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < n; s += stride) {
    for (int w = 0; w < nwords; ++w) t.keys[s * nwords + w] = kEmptyWord;
    t.rows[s] = 0;
    for (int a = 0; a < al.nacc; ++a) {
      uint64_t id = identity_bits(al.kind[a]);
      if (acc_bytes(al.kind[a]) == 4) reinterpret_cast<uint32_t*>(t.acc[a])[s] = static_cast<uint32_t>(id);
      else reinterpret_cast<uint64_t*>(t.acc[a])[s] = id;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *t.special_used = 0;
}

// ARG: the plan carries ARGMIN / ARGMAX accumulators.
template <int NW, bool ARG>
__global__ void k_agg_global(const __grid_constant__ Plan plan, const __grid_constant__ TableRef t, int64_t n, uint32_t max_probes)
{
  const Level<Global> G = global_level(t);
  const int64_t stride  = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    uint64_t k[NW];
    if (!pack_key<NW>(plan.key, r, k)) continue;
    int64_t g = global_slot<NW>(t, k, max_probes);
    if (g < 0) continue;
    accumulate_row<Global, ARG>(plan, G, g, r, t.status);
  }
}

// Per-CTA privatised aggregation.  Shared memory holds S+1 slots (slot S is
// the reserved all-ones key): keys, row counts and every accumulator array.
template <int NW, bool ARG>
__global__ void __launch_bounds__(512) k_agg_privatized(const __grid_constant__ Plan plan,
                                                        const __grid_constant__ TableRef t,
                                                        const __grid_constant__ SmemLayout sl,
                                                        int64_t n,
                                                        int64_t rows_per_block,
                                                        uint32_t smem_probes,
                                                        uint32_t max_probes)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t s_special;
  const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t S    = sl.slots;
  const Level<Shared> L{base, &sl};
  const uint32_t keys = base + sl.keys_off;

  // identity fill
  uint64_t* skeys = reinterpret_cast<uint64_t*>(smem + sl.keys_off);
  uint32_t* srows = reinterpret_cast<uint32_t*>(smem + sl.rows_off);
  for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) {
    for (int w = 0; w < NW; ++w) skeys[s * NW + w] = kEmptyWord;
    srows[s] = 0;
    for (int a = 0; a < plan.acc.nacc; ++a) {
      uint64_t id = identity_bits(plan.acc.kind[a]);
      if (acc_bytes(plan.acc.kind[a]) == 4) reinterpret_cast<uint32_t*>(smem + sl.acc_off[a])[s] = static_cast<uint32_t>(id);
      else reinterpret_cast<uint64_t*>(smem + sl.acc_off[a])[s] = id;
    }
  }
  if (threadIdx.x == 0) s_special = 0;
  __syncthreads();

  const Level<Global> G = global_level(t);
  const int64_t begin   = static_cast<int64_t>(blockIdx.x) * rows_per_block;
  const int64_t end     = min(n, begin + rows_per_block);
  for (int64_t r = begin + threadIdx.x; r < end; r += blockDim.x) {
    uint64_t k[NW];
    if (!pack_key<NW>(plan.key, r, k)) continue;
    int64_t s;
    if (key_is_empty<NW>(k)) {
      s = S;
      if (s_special == 0) s_special = 1;
    } else {
      s = find_or_insert<Shared, NW>(keys, S - 1, k, hash_key<NW>(k), smem_probes);
    }
    if (s >= 0) {
      accumulate_row<Shared, ARG>(plan, L, s, r, t.status);
    } else {
      int64_t g = global_slot<NW>(t, k, max_probes);
      if (g >= 0) accumulate_row<Global, ARG>(plan, G, g, r, t.status);
    }
  }
  __syncthreads();

  // flush the partial table into the global one
  for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) {
    uint64_t k[NW];
    for (int w = 0; w < NW; ++w) k[w] = skeys[s * NW + w];
    bool occupied = (s < S) ? !key_is_empty<NW>(k) : (s_special != 0);
    if (!occupied) continue;
    int64_t g = global_slot<NW>(t, k, max_probes);
    if (g >= 0) merge_slot<Shared, ARG>(plan, L, s, G, g, t.status);
  }
}

// Sampled distinct count: inserts a strided sample of packed keys (folded to
// 64 bits) into a small global set, counts first insertions and, per set
// slot, the sampled rows of its key.
template <int NW>
__global__ void k_sample_distinct(const __grid_constant__ KeyPlan kp,
                                  int64_t n,
                                  int64_t nsample,
                                  uint64_t* set,
                                  uint32_t* set_rows,
                                  uint64_t set_mask,
                                  unsigned long long* counters)
{
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nsample; i += stride) {
    int64_t r = static_cast<int64_t>((static_cast<double>(i) + 0.5) * static_cast<double>(n) / static_cast<double>(nsample));
    if (r >= n) r = n - 1;
    uint64_t k[NW];
    if (!pack_key<NW>(kp, r, k)) continue;
    atomicAdd(&counters[0], 1ULL);
    uint64_t f[1] = {hash_key<NW>(k)};
    if (f[0] == kEmptyWord) f[0] = 0;
    uint64_t s = fmix64(f[0] ^ 0x5bd1e995ULL) & set_mask;
    for (uint64_t p = 0; p <= set_mask; ++p) {
      uint64_t old = atomicCAS(reinterpret_cast<unsigned long long*>(set + s), kEmptyWord, f[0]);
      if (old == kEmptyWord) atomicAdd(&counters[1], 1ULL);
      if (old == kEmptyWord || old == f[0]) {
        atomicAdd(set_rows + s, 1u);
        break;
      }
      s = (s + 1) & set_mask;
    }
  }
}

// Keys sampled at least kHeavySample times: heavy[0] += their number,
// heavy[1] += their sampled rows.
__global__ void k_sample_heavy(const uint32_t* set_rows, uint64_t set_cap, unsigned long long* heavy)
{
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < set_cap; i += stride) {
    const uint32_t c = set_rows[i];
    if (c >= kHeavySample) {
      atomicAdd(&heavy[0], 1ULL);
      atomicAdd(&heavy[1], static_cast<unsigned long long>(c));
    }
  }
}

__global__ void k_fill_u64(uint64_t* p, uint64_t n, uint64_t v)
{
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}


// ------------------------------------------------------------- finalize

__device__ __forceinline__ void store_bits(void* p, int64_t i, int width, uint64_t v)
{
  switch (width) {
    case 1: reinterpret_cast<uint8_t*>(p)[i] = static_cast<uint8_t>(v); break;
    case 2: reinterpret_cast<uint16_t*>(p)[i] = static_cast<uint16_t>(v); break;
    case 4: reinterpret_cast<uint32_t*>(p)[i] = static_cast<uint32_t>(v); break;
    default: reinterpret_cast<uint64_t*>(p)[i] = v; break;
  }
}

__device__ __forceinline__ uint64_t ld_acc(const TableRef& t, int a, uint64_t s, int bytes)
{
  if (bytes == 4) return reinterpret_cast<const uint32_t*>(t.acc[a])[s];
  return reinterpret_cast<const uint64_t*>(t.acc[a])[s];
}

__global__ void k_finalize(const __grid_constant__ Plan plan, const __grid_constant__ TableRef t, const uint32_t* map, int64_t G, const __grid_constant__ OutPlan op)
{
  const int lane        = threadIdx.x & 31;
  const int64_t wstride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31); base < G;
       base += wstride) {
    const int64_t g    = base + lane;
    const bool active  = g < G;
    const uint64_t s   = active ? map[g] : 0;
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    uint64_t k[2]      = {0, 0};
    if (active) {
      for (int w = 0; w < plan.key.nwords; ++w) k[w] = t.keys[s * plan.key.nwords + w];
      if (s == t.cap) k[0] = k[1] = kEmptyWord;
    }
    // keys
    for (int c = 0; c < plan.key.ncols; ++c) {
      const KeyCol& kc = plan.key.cols[c];
      uint64_t word    = k[kc.word];
      bool valid       = true;
      if (kc.null_bit) valid = ((k[kc.null_word] >> kc.null_shift) & 1ULL) == 0;
      if (active) {
        int bits   = kc.width * 8;
        uint64_t v = (bits == 64) ? word : ((word >> kc.shift) & ((1ULL << bits) - 1));
        store_bits(op.key_data[c], g, kc.width, valid ? v : 0);
      }
      if (op.key_mask[c] != nullptr) {
        uint32_t bal = __ballot_sync(0xffffffffu, active && valid);
        if (lane == 0) {
          op.key_mask[c][base >> 5] = bal;
          uint32_t nulls = __popc(act & ~bal);
          if (nulls) atomicAdd(op.null_counts + c, static_cast<unsigned long long>(nulls));
        }
      }
    }
    // results (an output without data belongs to a sorted kind, written later)
    for (int o = 0; o < op.nout; ++o) {
      const OutCol& oc  = op.out[o];
      if (oc.data == nullptr) continue;
      const Channel& ch = plan.chan[oc.chan];
      bool valid        = false;
      uint64_t vbits    = 0;
      if (active) {
        uint32_t rows = t.rows[s];
        uint32_t cnt  = (ch.a_cnt >= 0) ? reinterpret_cast<const uint32_t*>(t.acc[ch.a_cnt])[s] : rows;
        valid         = cnt > 0;
        switch (oc.kind) {
          case GBX_AGG_COUNT_VALID: vbits = cnt; valid = true; break;
          case GBX_AGG_COUNT_ALL: vbits = rows; valid = true; break;
          case GBX_AGG_SUM:
          case GBX_AGG_SUM_OF_SQUARES:
          case GBX_AGG_PRODUCT: {
            int a = (oc.kind == GBX_AGG_SUM) ? ch.a_sum : (oc.kind == GBX_AGG_PRODUCT ? ch.a_prod : ch.a_sq);
            uint64_t raw = ld_acc(t, a, s, 8);
            if (ch.is_float) {
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
            bool mn      = oc.kind == GBX_AGG_MIN;
            int a        = mn ? ch.a_min : ch.a_max;
            uint64_t raw = ld_acc(t, a, s, minmax_is64(ch.ptype) ? 8 : 4);
            vbits        = dec_minmax(raw, ch.ptype, mn);
            break;
          }
          case GBX_AGG_ARGMIN:
          case GBX_AGG_ARGMAX: {
            // the row of the group's extreme value; null (data -1, the
            // reference's ARGMIN/ARGMAX_SENTINEL) when no value was valid
            bool mn = oc.kind == GBX_AGG_ARGMIN;
            int a   = mn ? ch.a_amin : ch.a_amax;
            uint32_t row;
            if (minmax_is64(ch.ptype)) {
              row = static_cast<uint32_t>(ld_acc(t, a, s, 4));
            } else {
              uint64_t w = ld_acc(t, a, s, 8);
              row        = (w == identity_bits(plan.acc.kind[a])) ? 0xffffffffu
                           : mn                                   ? static_cast<uint32_t>(w)
                                                                  : ~static_cast<uint32_t>(w);
            }
            valid = row != 0xffffffffu;
            vbits = row;
            break;
          }
          case GBX_AGG_MEAN: {
            if (!valid) break;
            uint64_t raw = ld_acc(t, ch.a_sum, s, 8);
            if (oc.out_ptype == P_F64) {
              // integer SUMs are INT64 (target_type), so the mean divides the
              // signed 64-bit sum, as binary_operation(DIV) does on it
              double sum = ch.is_float ? __longlong_as_double(static_cast<long long>(raw))
                                       : static_cast<double>(static_cast<int64_t>(raw));
              vbits = static_cast<uint64_t>(__double_as_longlong(sum / static_cast<double>(cnt)));
            } else {
              // duration / decimal MEAN: the SUM wraps to the source width, then
              // integer division (binary_operation DIV, hash/groupby.cu:298-304)
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
            uint64_t kb = ld_acc(t, ch.a_k, s, 8);
            double s2   = __longlong_as_double(static_cast<long long>(ld_acc(t, ch.a_s2, s, 8)));
            double var;
            if (kb == kShiftUnset) {
              var = s2;  // NaN inputs only
            } else {
              double K  = __longlong_as_double(static_cast<long long>(kb));
              double S1 = shifted_sum(ch.is_float, ch.ptype, ld_acc(t, ch.a_sum, s, 8),
                                      ch.a_s1 >= 0 ? ld_acc(t, ch.a_s1, s, 8) : 0, nn, K);
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
        const bool arg = oc.kind == GBX_AGG_ARGMIN || oc.kind == GBX_AGG_ARGMAX;
        store_bits(oc.data, g, oc.out_width, valid ? vbits : (arg ? 0xffffffffULL : 0));
      }
      if (oc.mask != nullptr) {
        uint32_t bal = __ballot_sync(0xffffffffu, active && valid);
        if (lane == 0) {
          oc.mask[base >> 5] = bal;
          uint32_t nulls = __popc(act & ~bal);
          if (nulls) atomicAdd(op.null_counts + kMaxKeyCols + o, static_cast<unsigned long long>(nulls));
        }
      }
    }
  }
}

// -------------------------------------------------------------- launchers

namespace {
inline int grid_for(int64_t work, int block, int max_blocks)
{
  int64_t b = (work + block - 1) / block;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return static_cast<int>(b);
}
}  // namespace

cudaError_t launch_init_table(const TableRef& t, const AccLayout& al, int nwords, int num_sms, cudaStream_t st)
{
  int grid = grid_for(static_cast<int64_t>(t.cap + 1), 256, num_sms * 16);
  k_init_table<<<grid, 256, 0, st>>>(t, al, nwords);
  return cudaGetLastError();
}

cudaError_t launch_sample(const KeyPlan& kp, int64_t n, int64_t nsample, uint64_t* set, uint32_t* set_rows,
                          uint64_t set_cap, unsigned long long* counters, unsigned long long* heavy, int num_sms,
                          cudaStream_t st)
{
  const int fill_grid = grid_for(static_cast<int64_t>(set_cap), 256, num_sms * 8);
  k_fill_u64<<<fill_grid, 256, 0, st>>>(set, set_cap, kEmptyWord);
  cudaError_t e = cudaMemsetAsync(set_rows, 0, set_cap * sizeof(uint32_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(heavy, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  int grid = grid_for(nsample, 256, num_sms * 8);
  if (kp.nwords == 1) k_sample_distinct<1><<<grid, 256, 0, st>>>(kp, n, nsample, set, set_rows, set_cap - 1, counters);
  else k_sample_distinct<2><<<grid, 256, 0, st>>>(kp, n, nsample, set, set_rows, set_cap - 1, counters);
  k_sample_heavy<<<fill_grid, 256, 0, st>>>(set_rows, set_cap, heavy);
  return cudaGetLastError();
}

cudaError_t launch_agg_global(const Plan& p, const TableRef& t, int64_t n, uint32_t max_probes, int num_sms,
                              cudaStream_t st)
{
  int grid       = grid_for(n, 256, num_sms * 8);
  const bool arg = plan_has_arg(p);
  if (p.key.nwords == 1) {
    if (arg) k_agg_global<1, true><<<grid, 256, 0, st>>>(p, t, n, max_probes);
    else k_agg_global<1, false><<<grid, 256, 0, st>>>(p, t, n, max_probes);
  } else {
    if (arg) k_agg_global<2, true><<<grid, 256, 0, st>>>(p, t, n, max_probes);
    else k_agg_global<2, false><<<grid, 256, 0, st>>>(p, t, n, max_probes);
  }
  return cudaGetLastError();
}

cudaError_t launch_agg_privatized(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int block,
                                  int grid, uint32_t smem_probes, uint32_t max_probes, cudaStream_t st)
{
  int64_t rpb = (n + grid - 1) / grid;
  auto run    = [&](auto kernel) -> cudaError_t {
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(kernel), sl.total);
    if (e != cudaSuccess) return e;
    kernel<<<grid, block, sl.total, st>>>(p, t, sl, n, rpb, smem_probes, max_probes);
    return cudaGetLastError();
  };
  const bool arg = plan_has_arg(p);
  if (p.key.nwords == 1) return arg ? run(k_agg_privatized<1, true>) : run(k_agg_privatized<1, false>);
  return arg ? run(k_agg_privatized<2, true>) : run(k_agg_privatized<2, false>);
}

cudaError_t launch_finalize(const Plan& p, const TableRef& t, const uint32_t* map, int64_t G, const OutPlan& op,
                            int num_sms, cudaStream_t st)
{
  if (G <= 0) return cudaSuccess;
  int grid = grid_for(G, 256, num_sms * 8);
  k_finalize<<<grid, 256, 0, st>>>(p, t, map, G, op);
  return cudaGetLastError();
}

}  // namespace gbx

namespace gbx {

// Valid-bit counts of several masks (one grid-stride sweep per mask).
__global__ void k_count_valid(const __grid_constant__ MaskSpans ms, unsigned long long* out)
{
  const int64_t tid    = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int c = 0; c < ms.n; ++c) {
    const MaskSpan sp = ms.span[c];
    const int64_t b0  = sp.offset;
    const int64_t b1  = sp.offset + sp.size;
    const int64_t w0  = b0 >> 5;
    const int64_t w1  = (b1 + 31) >> 5;
    unsigned long long local = 0;
    for (int64_t w = w0 + tid; w < w1; w += stride) {
      uint32_t word = __ldg(sp.mask + w);
      int64_t lo    = w << 5;
      if (lo < b0) word &= 0xffffffffu << (b0 - lo);
      if (lo + 32 > b1) word &= 0xffffffffu >> (lo + 32 - b1);
      local += __popc(word);
    }
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out + c, local);
  }
}

// dst bits [0, n) = src bits [src_bit, src_bit + n); every dst word of the
// range is written (bits past n cleared); src words are read only where
// their bits are needed.
__global__ void k_copy_bits(const uint32_t* __restrict__ src, int64_t src_bit, uint32_t* __restrict__ dst, int64_t n)
{
  const int64_t words  = (n + 31) >> 5;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < words; w += stride) {
    const int64_t b   = src_bit + (w << 5);
    const int64_t sw  = b >> 5;
    const int sh      = static_cast<int>(b & 31);
    const int64_t rem = n - (w << 5);
    uint32_t v        = __ldg(src + sw) >> sh;
    if (sh != 0 && rem > 32 - sh) v |= __ldg(src + sw + 1) << (32 - sh);
    if (rem < 32) v &= (1u << rem) - 1u;
    dst[w] = v;
  }
}

cudaError_t ensure_dynamic_smem(const void* func, size_t bytes)
{
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limit;
  int device    = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[{device, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e == cudaSuccess) cur = bytes;
  return e;
}

cudaError_t launch_copy_bits(const uint32_t* src, int64_t src_bit, uint32_t* dst, int64_t n, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  const int64_t words = (n + 31) >> 5;
  int64_t b           = (words + 255) / 256;
  if (b > 4096) b = 4096;
  k_copy_bits<<<static_cast<int>(b), 256, 0, st>>>(src, src_bit, dst, n);
  return cudaGetLastError();
}

cudaError_t launch_count_valid(const MaskSpans& ms, unsigned long long* out_valid, int num_sms, cudaStream_t st)
{
  if (ms.n == 0) return cudaSuccess;
  int64_t words = 0;
  for (int c = 0; c < ms.n; ++c) words = words > (ms.span[c].size / 32 + 2) ? words : (ms.span[c].size / 32 + 2);
  int64_t b = (words + 255) / 256;
  if (b < 1) b = 1;
  if (b > num_sms * 4) b = num_sms * 4;
  k_count_valid<<<static_cast<int>(b), 256, 0, st>>>(ms, out_valid);
  return cudaGetLastError();
}

}  // namespace gbx

namespace gbx {
// Loads the code of every kernel gbx_groupby_aggregate_noalloc can launch on
// the current device (cudaFuncGetAttributes loads a kernel that lazy module
// loading has not loaded yet), so that the call's first use on a device sets
// aside all of its device memory before it does any work.
cudaError_t load_noalloc_kernels()
{
  const void* kernels[] = {
    reinterpret_cast<const void*>(k_count_valid),
    reinterpret_cast<const void*>(k_init_table),
    reinterpret_cast<const void*>(k_agg_global<1, false>),
    reinterpret_cast<const void*>(k_agg_global<1, true>),
    reinterpret_cast<const void*>(k_agg_global<2, false>),
    reinterpret_cast<const void*>(k_agg_global<2, true>),
    compact_kernel(1),
    compact_kernel(2),
    reinterpret_cast<const void*>(k_finalize),
  };
  for (const void* k : kernels) {
    cudaFuncAttributes attr;
    const cudaError_t e = cudaFuncGetAttributes(&attr, k);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace gbx
