// gbx_kernels.hpp -- host-visible launch interface of libgbx's kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gbx.h"
#include "gbx_plan.hpp"

namespace gbx {

constexpr int kMaxOut = 64;

// Byte offsets of the per-CTA shared-memory table (S + 1 slots).
struct SmemLayout {
  uint32_t slots;  // S, power of two
  uint32_t keys_off;
  uint32_t rows_off;
  uint32_t acc_off[kMaxAccs];
  uint32_t total;
};

// One finalised output column.
struct OutCol {
  void* data;
  uint32_t* mask;   // nullptr: no null mask
  int32_t kind;     // gbx_agg_kind
  int32_t ddof;
  int8_t chan;
  int8_t out_ptype; // PhysType of the output element
  int8_t out_width; // bytes
  int8_t pad;
};

struct OutPlan {
  int32_t nout;
  unsigned long long* null_counts;  // [key columns..., outputs...] (zeroed by the caller)
  void* key_data[kMaxKeyCols];
  uint32_t* key_mask[kMaxKeyCols];
  OutCol out[kMaxOut];
};

cudaError_t launch_init_table(const TableRef& t, const AccLayout& al, int nwords, int num_sms, cudaStream_t st);
cudaError_t launch_sample(const KeyPlan& kp, int64_t n, int64_t nsample, uint64_t* set, uint64_t set_cap,
                          unsigned long long* counters, int num_sms, cudaStream_t st);
cudaError_t launch_agg_global(const Plan& p, const TableRef& t, int64_t n, uint32_t max_probes, int num_sms,
                              cudaStream_t st);
cudaError_t launch_agg_privatized(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int block,
                                  int grid, uint32_t smem_probes, uint32_t max_probes, cudaStream_t st);
// cub select of occupied slot ids; call once with temp == nullptr to size `temp_bytes`.
cudaError_t compact_occupied(const TableRef& t, int nwords, uint32_t* map, int64_t* num_selected, void* temp,
                             size_t* temp_bytes, cudaStream_t st);
cudaError_t launch_finalize(const Plan& p, const TableRef& t, const uint32_t* map, int64_t G, const OutPlan& op,
                            int num_sms, cudaStream_t st);

}  // namespace gbx

namespace gbx {
// Null counts of up to `ncols` masks over [offset, offset + size): writes
// size - popcount(valid bits) into out[i] (out zeroed by the caller).
struct MaskSpan {
  const uint32_t* mask;
  int64_t offset;
  int64_t size;
};
constexpr int kMaxMaskSpans = 24;
struct MaskSpans {
  int32_t n;
  MaskSpan span[kMaxMaskSpans];
};
cudaError_t launch_count_valid(const MaskSpans& ms, unsigned long long* out_valid, int num_sms, cudaStream_t st);
}  // namespace gbx
