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
// Sampled distinct count of nsample strided rows: counters[0] = sampled rows,
// counters[1] = their distinct keys; heavy[0] = keys sampled at least
// kHeavySample times, heavy[1] = their sampled rows.  `set` holds set_cap
// words and `set_rows` set_cap counts (set_cap a power of two).
constexpr uint32_t kHeavySample = 4;
cudaError_t launch_sample(const KeyPlan& kp, int64_t n, int64_t nsample, uint64_t* set, uint32_t* set_rows,
                          uint64_t set_cap, unsigned long long* counters, unsigned long long* heavy, int num_sms,
                          cudaStream_t st);
cudaError_t launch_agg_global(const Plan& p, const TableRef& t, int64_t n, uint32_t max_probes, int num_sms,
                              cudaStream_t st);
cudaError_t launch_agg_privatized(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int block,
                                  int grid, uint32_t smem_probes, uint32_t max_probes, cudaStream_t st);
// Per-CTA tables fed by tile-local grouping (gbx_tiled.cu), for tables where
// tiled_fits() (at most 1,024 slots, table and a tile's staged values within
// half an SM's shared memory).
bool tiled_fits(const SmemLayout& sl, int nchan);
// Streamed tiles grouped in shared memory (gbx_stream.cu): one packed key
// word, no ARGMIN/ARGMAX, a table of at most 4,096 slots.
bool stream_fits(const Plan& p, const SmemLayout& sl);
size_t stream_smem_bytes(const Plan& p, const SmemLayout& sl);
cudaError_t launch_agg_stream(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                              uint32_t smem_probes, uint32_t max_probes, cudaStream_t st);
cudaError_t launch_agg_tiled(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                             uint32_t smem_probes, uint32_t max_probes, cudaStream_t st);
// ---- radix-partitioned path
// Row-partitioned copies of the inputs: packed key words (SoA), each
// channel's resolved value bits, and a validity byte per row for channels
// with nulls (valid == nullptr otherwise).
struct PartCol {
  const void* vals;
  const uint8_t* valid;
  int32_t width;
  int32_t pad;
};
struct PartBufs {
  const uint64_t* keys[2];
  PartCol col[kMaxChannels];
};

struct PartPlan {
  int32_t bits;              // P = 2^bits buckets, bucket = top bits of the key hash
  int32_t shard_bits;        // each bucket's counter is split over 2^shard_bits warps' shards
  uint32_t slice_rows;       // rows per work item of a large bucket
  uint32_t* counts;          // [(P << shard_bits) + 1] rows per (bucket, shard) (last entry 0)
  uint32_t* offsets;         // [(P << shard_bits) + 1] exclusive scan of counts
  uint32_t* cursor;          // [P << shard_bits] scatter cursors (copy of offsets)
  uint32_t* nslices;         // [P + 1] slices of a bucket larger than slice_rows, else 0 (last entry 0)
  uint32_t* item_start;      // [P + 1] exclusive scan of nslices
  uint32_t* multi;           // [P + 1] 1 when a bucket has several items (last entry 0)
  uint32_t* region;          // [P + 1] exclusive scan of multi: region table of the bucket
  uint32_t* item_bucket;     // [items] bucket of each work item
  unsigned long long* item_counter;  // work-item dispenser (slices)
  unsigned long long* bucket_counter;  // bucket dispenser (whole buckets)
  unsigned long long* out_counter;   // output rows written so far
  uint32_t region_slots;     // slots per region table (= the warp table size)
  int32_t* status;           // device status word
  // [n], indexed by partitioned row: a whole bucket whose rows do not fit
  // its warp's or CTA's shared memory ranks them here (slot above the rank
  // within the slot: 16 rank bits for warp tables, 19 for CTA tables)
  uint32_t* rank_rec;
  // [n], indexed by output row: (first row, row count) of a whole bucket's
  // group in the group-ordered copies
  uint2* group_run;
};

// launch_agg_tiled over the bucket-ordered copies `in` of a radix
// partitioning (*n_rows rows, at most n): each CTA takes one contiguous run of
// tiles, so its table holds the groups of the few buckets that run covers.
cudaError_t launch_agg_tiled_part(const Plan& p, const TableRef& t, const SmemLayout& sl, const PartBufs& in,
                                  const uint32_t* n_rows, int64_t n, int num_sms, uint32_t smem_probes,
                                  uint32_t max_probes, cudaStream_t st);

cudaError_t launch_part_hist(const KeyPlan& kp, int64_t n, const PartPlan& pp, int num_sms, cudaStream_t st);
// counts -> offsets (unless offsets_ready), nslices, item_start, multi,
// region (device scans)
cudaError_t launch_part_layout(const PartPlan& pp, void* temp, size_t* temp_bytes, int num_sms, cudaStream_t st,
                               bool offsets_ready = false);
// offsets[b] = first row of bucket b (b <= P) of *n_rows rows already in
// bucket order (one word per key word in `keys`): the bucket offsets read off
// the partitioned copies, for unsharded counters.
cudaError_t launch_part_bounds(int nwords, const uint64_t* const* keys, const uint32_t* n_rows, int bits,
                               uint32_t* offsets, int num_sms, cudaStream_t st);
// item_bucket[item_start[b] + j] = b for every slice j of every bucket b
cudaError_t launch_part_items(const PartPlan& pp, int64_t n, int num_sms, cudaStream_t st);
cudaError_t launch_part_scatter(const Plan& p, int64_t n, const PartPlan& pp, const PartBufs& out, int num_sms,
                                cudaStream_t st);
// Radix partitioning into bucket order (gbx_radix.cu): the same result as
// launch_part_scatter for 2^bits buckets with unsharded counters, in
// ceil(bits / 8) coalesced passes that alternate between `dst` and `tmp`
// (same layout) and end in `dst`.  The rows kept (a null key under EXCLUDE
// drops a row) are written to *n_kept (device) after the first pass;
// `counts` and `offsets` hold part_radix_count_bytes(n) bytes each, `temp`
// part_radix_temp_bytes(n).  launch_part_radix_hist0 runs the first pass's
// tile histogram early (and adds every kept row to bucket_counts[its bucket]
// when that is set, zeroed by the caller); launch_part_radix is told so with
// hist0_done.
size_t part_radix_count_bytes(int64_t n);
cudaError_t part_radix_temp_bytes(int64_t n, size_t* temp_bytes);
cudaError_t launch_part_radix_hist0(const Plan& p, int64_t n, int bits, uint32_t* counts, uint32_t* bucket_counts,
                                    cudaStream_t st);
cudaError_t launch_part_radix(const Plan& p, int64_t n, int bits, uint32_t* n_kept, const PartBufs& dst,
                              const PartBufs& tmp, uint32_t* counts, uint32_t* offsets, void* temp,
                              size_t temp_bytes, int32_t* status, bool hist0_done, cudaStream_t st);
// Aggregates every bucket of at most slice_rows rows (S-slot warp tables)
// and writes its groups to `op`, the rows permuted into group order in
// `sorted` (the layout of `in`, overwritten; its key words hold rank
// records) and each group's run listed in pp.group_run (two launches:
// grouping, then one thread per group).
cudaError_t launch_part_ranked(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                               uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st);
// The same with one bucket per CTA at a time over one S-slot shared table
// (S a power of two in [256, 4096]; pp.slice_rows <= 2^19), for buckets of
// up to a few thousand groups.
cudaError_t launch_part_ranked_cta(const Plan& p, const PartPlan& pp, const PartBufs& in, const PartBufs& sorted,
                                   uint32_t S, const OutPlan& op, int num_sms, cudaStream_t st);
// Aggregates the slices of the larger buckets (item_start[P] of them, > 0)
// into region tables of `t` (t.cap = regions * region_slots) that
// launch_part_region_finalize then writes out.
cudaError_t launch_part_agg(const Plan& p, const PartPlan& pp, const PartBufs& in, const TableRef& t,
                            const SmemLayout& sl, int num_sms, cudaStream_t st);
cudaError_t launch_part_region_finalize(const Plan& p, const PartPlan& pp, const TableRef& t, const OutPlan& op,
                                       int num_sms, cudaStream_t st);

// Warp-private shared-memory tables (sl describes one warp's table).
cudaError_t launch_agg_warp(const Plan& p, const TableRef& t, const SmemLayout& sl, int64_t n, int num_sms,
                            uint32_t max_probes, cudaStream_t st);
// Occupied slot ids of `t` into map[0, *num_selected) in unspecified order
// (gbx_scan.cu; *num_selected is zeroed first, on the stream).
cudaError_t compact_occupied(const TableRef& t, int nwords, uint32_t* map, int64_t* num_selected, int num_sms,
                             cudaStream_t st);
// The compaction kernel for `nwords` key words (to load it ahead of use).
const void* compact_kernel(int nwords);
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

// dst bits [0, n) = src bits [src_bit, src_bit + n) (a bitmask slice).
cudaError_t launch_copy_bits(const uint32_t* src, int64_t src_bit, uint32_t* dst, int64_t n, cudaStream_t st);

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`.  It never lowers it, so a launch on another thread that was
// sized against the current limit stays valid.
cudaError_t ensure_dynamic_smem(const void* func, size_t bytes);
}  // namespace gbx
