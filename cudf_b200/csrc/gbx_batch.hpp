// gbx_batch.hpp -- descriptors and launchers of the batched groupby: many
// independent groupby instances (same key / value types and aggregations,
// their own columns and row counts) aggregated by one persistent kernel.
//
// Every instance i owns
//   * its column buffers (InstCols; the element layout comes from the batch's
//     schema Plan, which all instances share);
//   * a global open-addressing table carved from one arena (TableRef);
//   * a mode chosen by the autotuner: a CTA-shared table in shared memory, a
//     shared-memory table per warp, or direct updates of the global table;
//   * a run of output rows [offset_i, offset_i + groups_i) in the batch's
//     concatenated output columns.
// The row ranges of all instances are cut into work items (tiles) that the
// persistent kernel's CTAs claim from a counter, largest first.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gbx_kernels.hpp"
#include "gbx_plan.hpp"

namespace gbx {

enum BatchMode : int32_t { BM_SHARED = 1, BM_WARP = 2, BM_GLOBAL = 3 };

// Dynamic shared memory limit set once on the aggregation kernel, so that a
// graph captured with any size up to it stays launchable.
constexpr size_t kBatchMaxDynamicSmem = 200 * 1024;

struct InstKeyCol {
  const void* data;
  const uint32_t* mask;  // nullptr: no nulls
  int64_t offset;
};

struct InstChan {
  const void* data;       // values (or dictionary indices)
  const uint32_t* mask;
  int64_t offset;
  const void* dict_data;  // dictionary keys (nullptr: plain column)
  int64_t dict_offset;
  int64_t dict_size;
};

struct InstCols {
  InstKeyCol key[kMaxKeyCols];
  InstChan chan[kMaxChannels];
};

// One instance as the kernels see it (device memory, 16-byte multiple so the
// persistent kernel copies it to shared memory with vector loads).
struct alignas(16) BatchInst {
  InstCols cols;
  TableRef t;      // its global table (status and special flag per instance)
  SmemLayout sl;   // its shared-memory table (BM_SHARED: one per CTA; BM_WARP: one per warp)
  int64_t num_rows;
  int32_t mode;    // BatchMode
  int32_t pad;
};

struct BatchItem {
  uint32_t inst;
  uint32_t pad;
  int64_t begin;
  int64_t end;
};

// Launchers (gbx_batch.cu).

// Per instance: the number of valid sampled rows (out[2i]) and how many
// distinct keys they hold (out[2i+1]), from up to `per_inst` evenly spaced rows.
cudaError_t launch_batch_sample(const Plan& schema, const BatchInst* insts, int ninst, int per_inst,
                                uint32_t* out, cudaStream_t st);

// Identity fill of every instance's global table.
cudaError_t launch_batch_init(const Plan& schema, const BatchInst* insts, int ninst, cudaStream_t st);

// The persistent aggregation kernel over `nitems` items (claimed through
// *counter, which must be zero).  `block` is 256 or 512; `grid` CTAs with
// `smem` bytes of dynamic shared memory each (batch_agg_max_grid first).
cudaError_t launch_batch_agg(const Plan& schema, const BatchInst* insts, const BatchItem* items, uint32_t nitems,
                             uint32_t* counter, int block, int grid, size_t smem, cudaStream_t st);

// Raises the aggregation kernel's shared-memory limit and returns the
// largest grid that is resident at once with `smem` bytes per CTA.
cudaError_t batch_agg_max_grid(const Plan& schema, int block, size_t smem, int num_sms, int* grid);

// Occupied slots per instance into counts[0..ninst), counts[ninst] = 0; then
// offsets = exclusive scan of counts (ninst + 1 entries).  `temp` of
// *temp_bytes bytes (query with temp == nullptr).
cudaError_t launch_batch_count(const Plan& schema, const BatchInst* insts, int ninst, int64_t* counts,
                               int64_t* offsets, void* temp, size_t* temp_bytes, cudaStream_t st);

// Writes every instance's groups to rows [offsets[i], offsets[i+1]) of the
// output columns (keys decoded, results finalised, validity or-ed into
// zeroed masks, null counts added to op.null_counts).
cudaError_t launch_batch_write(const Plan& schema, const BatchInst* insts, int ninst, const int64_t* offsets,
                               const OutPlan& op, cudaStream_t st);

}  // namespace gbx
