// gbx_sort.hpp -- MEDIAN, QUANTILE, NUNIQUE and NTH_ELEMENT over the groups
// of a finished hash table (gbx_sort.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "gbx_plan.hpp"

namespace gbx {

struct Scratch;

// One output column of a sorted kind.
struct SortedOut {
  int32_t kind;
  int32_t chan;                    // value channel of the plan
  int32_t null_policy;             // NUNIQUE, NTH_ELEMENT
  int32_t interpolation;           // QUANTILE (MEDIAN: LINEAR)
  int32_t num_quantiles;           // QUANTILE (MEDIAN: 1)
  int32_t out_width;               // NTH_ELEMENT: bytes of an output element
  int64_t nth;                     // NTH_ELEMENT
  const double* quantiles_dev;     // QUANTILE / MEDIAN: device array of num_quantiles
  void* data;                      // G (QUANTILE: G * num_quantiles) elements
  uint32_t* mask;                  // nullptr for NUNIQUE
  unsigned long long* null_count;  // device counter, zero on entry
};

struct SortedKindsArgs {
  Plan plan;
  TableRef table;
  const uint32_t* map;  // output row g -> table slot (the compacted occupied slots)
  int64_t num_groups;
  int64_t n;            // rows
  uint32_t max_probes;  // probe limit the table was built with
  std::vector<SortedOut> outs;  // one channel's MEDIAN / QUANTILE / NUNIQUE together
  Scratch* scratch;
  int32_t* status;
  int num_sms;
  cudaStream_t stream;
};

// Writes every output of `a.outs`, stream-ordered, without synchronising;
// the kernels launched are added to *launches.
void sorted_kinds(const SortedKindsArgs& a, int* launches);

}  // namespace gbx
