/*
 * gbx.h -- C ABI of libgbx, a B200 (sm_100a) hash groupby-aggregation library.
 *
 * This is the drop-in boundary for libcudf's hash groupby path:
 *   cudf::groupby::groupby(keys, null_policy, sorted).aggregate(requests, stream, mr)
 * (reference: cpp/include/cudf/groupby.hpp:96-199, cpp/src/groupby/groupby.cu:197-221,
 *  cpp/src/groupby/hash/groupby.cu:548-667).
 *
 * Every entry point takes plain pointers and sizes; no CUDA, C++ or torch types
 * appear in the signatures (a CUDA stream is passed as `void*`, i.e. a
 * cudaStream_t). All device pointers are CUDA device (or managed) memory on the
 * current device.  The header-only C++ facade under include/cudf/ rebuilds the
 * reference's C++ API on top of these functions.
 *
 * Error convention: every function returning `int` returns GBX_OK (0) or a
 * gbx_status code; the message of the last failure on the calling thread is
 * returned by gbx_last_error().  GBX_ERR_LOGIC corresponds to the reference's
 * cudf::logic_error (CUDF_EXPECTS / CUDF_FAIL, cpp/include/cudf/utilities/error.hpp:64),
 * GBX_ERR_CUDA to cudf::cuda_error (error.hpp:92), GBX_ERR_ALLOC to rmm::bad_alloc.
 */
#ifndef GBX_H
#define GBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBX_ABI_VERSION 5

#if defined(__GNUC__)
#define GBX_API __attribute__((visibility("default")))
#else
#define GBX_API
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum gbx_status {
  GBX_OK              = 0,
  GBX_ERR_LOGIC       = 1, /* invalid argument: cudf::logic_error */
  GBX_ERR_CUDA        = 2, /* CUDA runtime failure: cudf::cuda_error */
  GBX_ERR_ALLOC       = 3, /* device allocation failed: rmm::bad_alloc */
  GBX_ERR_UNSUPPORTED = 4, /* valid in libcudf, but not provided here (a type or kind of its sort-based path) */
  GBX_ERR_DEVICE      = 5  /* a bounded device-side loop gave up (status word set by a kernel) */
} gbx_status;

/* ---- types: numbering is cudf::type_id (cpp/include/cudf/types.hpp:203-235) ---- */
typedef enum gbx_type_id {
  GBX_TYPE_EMPTY = 0,
  GBX_TYPE_INT8,
  GBX_TYPE_INT16,
  GBX_TYPE_INT32,
  GBX_TYPE_INT64,
  GBX_TYPE_UINT8,
  GBX_TYPE_UINT16,
  GBX_TYPE_UINT32,
  GBX_TYPE_UINT64,
  GBX_TYPE_FLOAT32,
  GBX_TYPE_FLOAT64,
  GBX_TYPE_BOOL8,
  GBX_TYPE_TIMESTAMP_DAYS,
  GBX_TYPE_TIMESTAMP_SECONDS,
  GBX_TYPE_TIMESTAMP_MILLISECONDS,
  GBX_TYPE_TIMESTAMP_MICROSECONDS,
  GBX_TYPE_TIMESTAMP_NANOSECONDS,
  GBX_TYPE_DURATION_DAYS,
  GBX_TYPE_DURATION_SECONDS,
  GBX_TYPE_DURATION_MILLISECONDS,
  GBX_TYPE_DURATION_MICROSECONDS,
  GBX_TYPE_DURATION_NANOSECONDS,
  GBX_TYPE_DICTIONARY32,
  GBX_TYPE_STRING,
  GBX_TYPE_LIST,
  GBX_TYPE_DECIMAL32,
  GBX_TYPE_DECIMAL64,
  GBX_TYPE_DECIMAL128,
  GBX_TYPE_STRUCT,
  GBX_TYPE_NUM_TYPE_IDS
} gbx_type_id;

/* ---- aggregation kinds: numbering is cudf::aggregation::Kind
 *      (cpp/include/cudf/aggregation.hpp:86-124) ---- */
typedef enum gbx_agg_kind {
  GBX_AGG_SUM            = 0,
  GBX_AGG_PRODUCT        = 1,
  GBX_AGG_MIN            = 2,
  GBX_AGG_MAX            = 3,
  GBX_AGG_COUNT_VALID    = 4,
  GBX_AGG_COUNT_ALL      = 5,
  GBX_AGG_ANY            = 6,
  GBX_AGG_ALL            = 7,
  GBX_AGG_SUM_OF_SQUARES = 8,
  GBX_AGG_MEAN           = 9,
  GBX_AGG_M2             = 10,
  GBX_AGG_VARIANCE       = 11,
  GBX_AGG_STD            = 12,
  GBX_AGG_MEDIAN         = 13,
  GBX_AGG_QUANTILE       = 14,
  GBX_AGG_ARGMAX         = 15,
  GBX_AGG_ARGMIN         = 16,
  GBX_AGG_NUNIQUE        = 17,
  GBX_AGG_NTH_ELEMENT    = 18
  /* later kinds exist in libcudf; none of them is hash-computable */
} gbx_agg_kind;

/* cudf::null_policy (types.hpp:126) */
#define GBX_NULL_EXCLUDE 0
#define GBX_NULL_INCLUDE 1

/* ---- column / table views (borrowed, non-owning) ------------------------
 * Mirrors cudf::column_view: `data` points at row 0 of the underlying buffer,
 * `offset` is the view's first row (applied to `data` and to `null_mask`).
 * `null_mask` follows cudf's bitmask layout: 32-bit words, bit (i % 32) of
 * word (i / 32) set <=> row i valid; NULL means every row is valid.
 * For DICTIONARY32 columns `data` holds the indices (of integer type
 * `index_type_id`, default INT32) and `dict_keys` the dictionary's keys column;
 * `null_mask` is the dictionary's own mask.  DECIMAL32/64 carry `scale`.
 * For STRING key columns `data` holds the UTF-8 characters and `dict_keys`
 * the offsets column (INT32 or INT64, at least offset + size + 1 rows; row r's
 * characters are data[offsets[offset + r]] up to offsets[offset + r + 1]), as
 * a cudf strings column holds its offsets child.
 * For STRUCT key columns `dict_keys` points to an array of `num_children`
 * member views (fixed-width, STRING or STRUCT; not DICTIONARY32) and `data`
 * is unused; row r of the struct is row offset + r of every member (each
 * member applying its own offset too), as a cudf structs column holds its
 * children; members hold at least offset + size rows.  `num_children` is 0
 * for every other type.
 * `null_count` may be -1 (unknown): the library then counts nulls itself.
 */
typedef struct gbx_column_view {
  int32_t type_id;
  int32_t scale;
  int64_t size;
  int64_t offset;
  const void* data;
  const uint32_t* null_mask;
  int64_t null_count;
  int32_t index_type_id;
  int32_t num_children;
  const struct gbx_column_view* dict_keys;
} gbx_column_view;

typedef struct gbx_table_view {
  int32_t num_columns;
  int32_t reserved0;
  const gbx_column_view* columns;
} gbx_table_view;

/* cudf::interpolation (types.hpp:192-198), for QUANTILE. */
typedef enum gbx_interpolation {
  GBX_INTERP_LINEAR   = 0,
  GBX_INTERP_LOWER    = 1,
  GBX_INTERP_HIGHER   = 2,
  GBX_INTERP_MIDPOINT = 3,
  GBX_INTERP_NEAREST  = 4
} gbx_interpolation;

/* One aggregation of a request (cudf::groupby_aggregation).  `ddof` is used by
 * VARIANCE/STD (make_variance_aggregation(ddof), aggregation.hpp:311-337) and
 * holds n for NTH_ELEMENT (make_nth_element_aggregation(n, null_handling),
 * aggregation.hpp:410-411).  COUNT's null_policy is encoded in the kind:
 * COUNT_VALID (EXCLUDE) or COUNT_ALL (INCLUDE), as make_count_aggregation does
 * (aggregation.cpp:494-499); NUNIQUE and NTH_ELEMENT carry theirs in
 * `null_policy` (GBX_NULL_EXCLUDE / GBX_NULL_INCLUDE).  QUANTILE takes
 * `num_quantiles` values from the host array `quantiles` (clamped to [0, 1])
 * and an `interpolation` (make_quantile_aggregation, aggregation.hpp:364); its
 * result column holds num_groups * num_quantiles rows, group by group.
 * Fields a kind does not use are ignored (zero-initialise them). */
typedef struct gbx_aggregation {
  int32_t kind;
  int32_t ddof;
  int32_t null_policy;
  int32_t interpolation;
  int32_t num_quantiles;
  int32_t reserved0;
  const double* quantiles;
} gbx_aggregation;

/* cudf::groupby::aggregation_request (groupby.hpp:61-64). */
typedef struct gbx_request {
  gbx_column_view values;
  int32_t num_aggregations;
  int32_t reserved0;
  const gbx_aggregation* aggregations;
} gbx_request;

/* Stream-ordered device allocator (rmm::device_async_resource_ref).
 * `stream` is a cudaStream_t.  Pass NULL to use cudaMallocAsync/cudaFreeAsync. */
typedef struct gbx_allocator {
  void* ctx;
  void* (*allocate)(void* ctx, size_t bytes, void* stream);
  void (*deallocate)(void* ctx, void* ptr, size_t bytes, void* stream);
} gbx_allocator;

/* ---- owning results ------------------------------------------------------
 * An output column.  `view` describes it (data/null_mask point at the owned
 * buffers); a DICTIONARY32 key column borrows `dict_keys` from the input.
 * `null_mask` is NULL when the column has no mask (no nulls possible). */
typedef struct gbx_column {
  gbx_column_view view;
  void* data;
  uint32_t* null_mask;
  size_t data_bytes;
  size_t mask_bytes;
} gbx_column;

/* cudf::groupby::aggregation_result (groupby.hpp:88-91): one column per
 * requested aggregation, in request order. */
typedef struct gbx_aggregation_result {
  int32_t num_results;
  int32_t reserved0;
  gbx_column* results;
} gbx_aggregation_result;

/* The pair<unique_ptr<table>, vector<aggregation_result>> of aggregate(). */
typedef struct gbx_result {
  int64_t num_groups;
  int32_t num_key_columns;
  int32_t num_requests;
  gbx_column* keys;
  gbx_aggregation_result* requests;
  void* internal; /* allocator + stream used for release */
} gbx_result;

typedef struct gbx_groupby gbx_groupby;

/* ---- the plain groupby (the drop-in path) -------------------------------- */

/* cudf::groupby::groupby::groupby (groupby.hpp:128-132, groupby.cu:53-64).
 * Copies the key descriptors (not the data: the caller keeps `keys` alive, as
 * with the reference).  `keys_are_sorted` 0 (sorted::NO): one group per key,
 * in no particular order.  1 (sorted::YES): the caller declares the rows
 * sorted by key, and groups follow the reference's sort path
 * (sort_helper.cu:64-71, 96-104, 141-179): each run of equal adjacent rows is
 * a group (nulls equal, NaNs equal; under INCLUDE a null run between runs is
 * a group of its own), output in row order; under EXCLUDE with null keys the
 * reference sorts the rows again, and here every key is one group, output in
 * the order of each key's first row (the same order when the keys are
 * ascending).  Any other value fails with GBX_ERR_LOGIC. */
GBX_API int gbx_groupby_create(const gbx_table_view* keys,
                       int32_t null_policy,
                       int32_t keys_are_sorted,
                       gbx_groupby** out);

/* cudf::groupby::groupby::aggregate (groupby.hpp:187-199, groupby.cu:197-221).
 * Validates requests (size mismatch and invalid type/aggregation combinations
 * fail with GBX_ERR_LOGIC, like CUDF_EXPECTS), runs the hash path on `stream`
 * and returns owning results allocated from `mr` (NULL: cudaMallocAsync).
 * Synchronises `stream` once, to learn the number of groups (the reference's
 * retrieve_all does the same).  STRING, STRUCT, LIST and DECIMAL128 value
 * columns take COUNT_VALID / COUNT_ALL (their rows' validity), and STRING
 * values MIN / MAX too (a STRING result, byte order, null for a group with
 * no valid value; not with keys_are_sorted 1); other kinds over them are
 * GBX_ERR_UNSUPPORTED (libcudf's sort path).  On success *out must be freed
 * with gbx_result_release. */
GBX_API int gbx_groupby_aggregate(gbx_groupby* gb,
                          const gbx_request* requests,
                          int32_t num_requests,
                          void* stream,
                          const gbx_allocator* mr,
                          gbx_result** out);

/* Whether every request is computable by the hash path
 * (can_use_hash_groupby, hash/groupby.cu:635-651).  Returns 1/0, or -1 with
 * gbx_last_error() set on malformed input.  A 0 does not mean that
 * gbx_groupby_aggregate refuses the requests: M2, MEDIAN, QUANTILE, NUNIQUE
 * and NTH_ELEMENT, which libcudf computes on its sort path, are computed
 * here from the hash table's groups (the group order of the output is the
 * hash path's either way). */
GBX_API int gbx_can_use_hash_groupby(const gbx_request* requests, int32_t num_requests);

/* Output type of aggregation `kind` over a column of `type_id`
 * (cudf::detail::target_type, detail/aggregation/aggregation.hpp:1212-1367)
 * for the kinds gbx_groupby_aggregate computes; returns GBX_TYPE_EMPTY when
 * the combination is invalid or the kind is not computed here. */
GBX_API int32_t gbx_target_type(int32_t type_id, int32_t kind);

GBX_API void gbx_result_release(gbx_result* result);
GBX_API void gbx_groupby_destroy(gbx_groupby* gb);

/* Thread-local message of the last failure on this thread ("" if none). */
GBX_API const char* gbx_last_error(void);
GBX_API int32_t gbx_abi_version(void);

/* ---- tuning / introspection -------------------------------------------- */

/* Strategy the plain path uses for the aggregation pass. */
typedef enum gbx_strategy {
  GBX_STRATEGY_AUTO       = 0, /* chosen from a sampled cardinality estimate */
  GBX_STRATEGY_PRIVATIZED = 1, /* per-CTA shared-memory tables, flushed to a global table */
  GBX_STRATEGY_GLOBAL     = 2, /* every row updates the global open-addressing table */
  GBX_STRATEGY_PARTITIONED = 3, /* radix-partition rows by key hash, then per-partition smem tables */
  GBX_STRATEGY_WARP       = 4, /* per-warp private shared-memory tables, no atomics on the hot path */
  GBX_STRATEGY_BUCKETED   = 5  /* radix-partition rows into 2^8 or 2^16 buckets, then group tiles of the
                                  bucket-ordered rows in per-CTA shared-memory tables, flushed to a global table */
} gbx_strategy;

/* Force a strategy for subsequent calls on this gb object (AUTO restores). */
GBX_API int gbx_groupby_set_strategy(gbx_groupby* gb, int32_t strategy);

/* Statistics of the last aggregate() call on `gb` (host-side record). */
typedef struct gbx_stats {
  int64_t num_rows;
  int64_t num_groups;
  int64_t estimated_groups;
  int64_t table_capacity;
  int32_t strategy;      /* gbx_strategy actually used */
  int32_t retries;       /* table re-sizes after an overflow */
  int64_t scratch_bytes; /* device scratch held during the call */
  int32_t kernel_launches;
  int32_t timed;         /* 1 when the phase times below were recorded */
  /* CUDA-event times on the call's stream (gbx_groupby_set_timing) in ms */
  float sample_ms;       /* null counts + sampled distinct count */
  float init_ms;         /* table identity fill (0 for the partitioned strategy) */
  float aggregate_ms;    /* the aggregation pass over the rows */
  float compact_ms;      /* occupied-slot compaction */
  float finalize_ms;     /* output keys/results + null counts */
  float total_ms;        /* first to last event of the call */
  /* partitioned strategy: log2 of the bucket count and the slots of each
   * bucket's grouping table (a warp's, or, with buckets of a few thousand
   * groups, a CTA's); 0 for the other strategies */
  int32_t partition_bits;
  int32_t bucket_slots;
  float partition_ms;    /* partitioned strategy: the radix partition passes (else 0) */
  int32_t reserved1;
} gbx_stats;

GBX_API int gbx_groupby_last_stats(const gbx_groupby* gb, gbx_stats* out);

/* Record per-phase CUDA-event times into gbx_stats on subsequent calls
 * (enable = 1) or stop (0).  Adds a few event records per call. */
GBX_API int gbx_groupby_set_timing(gbx_groupby* gb, int32_t enable);

/* ---- groupby without device allocation -----------------------------------
 * No counterpart in the reference (libcudf always allocates its hash set and
 * results from an rmm resource).
 *
 * For callers that cannot allocate device memory during the call: an engine
 * that gives its whole GPU budget to its own pool and forbids other
 * allocations, or a latency-critical thread on which cudaMalloc / cudaFree
 * would block or synchronise the device.  This call computes the same result
 * as gbx_groupby_aggregate but allocates nothing: the hash table, compaction
 * map and control words live in a fixed device array of
 * GBX_NOALLOC_SCRATCH_BYTES inside libgbx, and the caller passes every output
 * buffer.
 *
 * Set-up: each call looks up the array's device address on the current
 * device.  Under CUDA's lazy module loading (the default) the array and the
 * code of the kernels this call launches reach the device only when first
 * used; the first call on a device (in a CUDA context) loads all of them
 * before it does any work, and the array then stays on that device until the
 * process exits or the device is reset.  A caller that hands the GPU's memory
 * to its own pool makes that first call beforehand -- an input of zero rows
 * does the set-up and nothing else -- or runs with CUDA_MODULE_LOADING=EAGER.
 *
 * Limits: at most GBX_NOALLOC_MAX_GROUPS groups (more is rejected with
 * GBX_ERR_LOGIC after the aggregation pass, outputs untouched), and the
 * aggregations' per-group state must fit the array (else GBX_ERR_LOGIC).
 * MEDIAN, QUANTILE, NUNIQUE and NTH_ELEMENT, which sort every row, STRING
 * keys and keys beyond 128 packed bits, and a groupby created with
 * keys_are_sorted 1, which label every row first, are refused with
 * GBX_ERR_UNSUPPORTED.
 *
 * Outputs: `out_keys` has one gbx_column per key column and `out_results` one
 * per aggregation of every request, in request order.  The caller sets each
 * column's `data` and `null_mask` (room for `capacity` bits in 32-bit words;
 * required where the output can hold nulls, ignored otherwise); the call
 * fills each `view` and `*num_groups`.  A result column's `data` holds
 * `capacity` rows of gbx_target_type(value type, kind); a key column's holds
 * `capacity` rows of the key column's own type -- for a DICTIONARY32 key,
 * rows of its index type (index_type_id, up to 8 bytes), as the output key
 * is a dictionary column over the input's keys.
 *
 * Every call shares the one array: calls whose work overlaps on the GPU (on
 * different streams or threads) race and corrupt each other's results, so
 * serialise them.  The array keeps the last call's contents; each call clears
 * what must start at zero itself.  The call synchronises `stream` up to three
 * times: after counting nulls (only when some column's null_count is -1),
 * after the aggregation pass (to learn the group count) and after writing
 * the outputs (to report their null counts). */
#define GBX_NOALLOC_SCRATCH_BYTES (16u << 20)
#define GBX_NOALLOC_MAX_GROUPS 32768
GBX_API int gbx_groupby_aggregate_noalloc(gbx_groupby* gb,
                                          const gbx_request* requests,
                                          int32_t num_requests,
                                          void* stream,
                                          gbx_column* out_keys,
                                          gbx_column* out_results,
                                          int64_t capacity,
                                          int64_t* num_groups);

/* ---- batched groupby ------------------------------------------------------
 * No counterpart in the reference: a libcudf caller with many tables loops
 * over cudf::groupby::groupby(keys_i).aggregate(requests_i), one call (with
 * its own launches, allocations and result-size synchronisation) per table.
 *
 * A batch holds many independent groupby instances that share one schema:
 * the same number and types of key columns, and the same requests (value
 * types, aggregation kinds and ddof) over each instance's own columns and row
 * count.  gbx_batch_create samples every instance's distinct count, lets the
 * autotuner choose per instance a table mode (shared-memory table per CTA,
 * per warp, or the global table), its table sizes and tile size, and the
 * block shape of the batch; it then allocates one table arena and the
 * outputs and captures the whole batch -- table fill, one persistent
 * aggregation kernel over all instances' tiles, group counting, offsets and
 * output writing -- as one CUDA graph.  gbx_batch_execute launches that
 * graph (one launch) and waits for it.
 *
 * Inputs are read at execute time from the buffers given at create (or the
 * last gbx_batch_rebind): the caller may refill them in place between
 * executes.  Results are the concatenation of every instance's groups:
 * instance i's groups are rows [group_offsets[i], group_offsets[i+1]) of the
 * output columns, in unspecified order within the run, with the same values
 * (and the same dtypes) as gbx_groupby_aggregate on that instance alone.  A
 * result column carries a null mask when any instance's output can hold
 * nulls.  The output columns belong to the batch and stay valid until the
 * next execute, rebind or destroy. */
typedef struct gbx_batch gbx_batch;

typedef struct gbx_batch_instance {
  gbx_table_view keys;          /* this instance's key columns */
  const gbx_request* requests;  /* num_requests requests over this instance's rows */
} gbx_batch_instance;

typedef enum gbx_batch_mode {
  GBX_BATCH_MODE_AUTO   = 0, /* the autotuner's choice per instance */
  GBX_BATCH_MODE_SHARED = 1, /* one shared-memory table per CTA, merged into the global table */
  GBX_BATCH_MODE_WARP   = 2, /* one shared-memory table per warp, updated without atomics */
  GBX_BATCH_MODE_GLOBAL = 3  /* every row updates the instance's global table */
} gbx_batch_mode;

typedef enum gbx_batch_tune {
  GBX_TUNE_OFF     = 0, /* built-in defaults; the tuning file is not read */
  GBX_TUNE_CACHED  = 1, /* choices from the tuning file where present, defaults elsewhere */
  GBX_TUNE_MISSING = 2, /* as CACHED, and measure + append the classes the file lacks */
  GBX_TUNE_ALL     = 3  /* re-measure every class present in the batch and append */
} gbx_batch_tune;

typedef struct gbx_batch_options {
  int32_t null_policy;         /* GBX_NULL_EXCLUDE or GBX_NULL_INCLUDE, for every instance */
  int32_t tune;                /* gbx_batch_tune */
  const char* tune_file;       /* the persisted tuning table (NULL: none) */
  int32_t force_mode;          /* gbx_batch_mode for every instance (AUTO: per instance) */
  int32_t block_threads;       /* 0: tuner's choice; else 256 or 512 */
  int32_t one_shot;            /* 1: launch the kernels directly at execute instead of capturing a
                                  graph (cheaper for a batch that runs once) */
  int64_t tile_rows;           /* 0: tuner's choice; else rows per work item */
} gbx_batch_options;

typedef struct gbx_batch_output {
  int32_t num_instances;
  int32_t reserved;
  const int64_t* group_offsets;        /* host memory, num_instances + 1 entries */
  const int64_t* device_group_offsets; /* the same offsets in device memory */
  gbx_result columns;                  /* concatenated keys and results (owned by the batch) */
} gbx_batch_output;

typedef struct gbx_batch_stats {
  int32_t num_instances;
  int32_t block_threads;       /* threads per CTA of the aggregation kernel */
  int32_t grid;                /* persistent CTAs */
  int32_t work_items;
  int64_t num_rows;            /* all instances */
  int64_t num_groups;          /* last execute */
  int64_t dynamic_smem;        /* bytes per CTA */
  int64_t arena_bytes;         /* global tables */
  int64_t output_rows;         /* capacity of the concatenated outputs */
  int32_t mode_count[4];       /* instances per gbx_batch_mode (index 0 unused) */
  int32_t classes;             /* tuning classes present */
  int32_t classes_measured;    /* measured by this create */
  int32_t classes_cached;      /* read from the tuning file */
  int32_t retries;             /* re-plans after a table overflow */
  int32_t graph_nodes;
  int32_t kernels_per_execute; /* kernel launches per execute */
  float create_ms;             /* host wall time of gbx_batch_create */
  float tune_ms;               /* of which measuring candidates */
  float execute_ms;            /* CUDA-event time of the last execute's launch */
  float init_ms;               /* of which: table fill (events recorded by the execution) */
  float aggregate_ms;          /*   the persistent aggregation kernel */
  float output_ms;             /*   counting, offsets and output writing */
} gbx_batch_stats;

GBX_API int gbx_batch_create(const gbx_batch_instance* instances,
                             int32_t num_instances,
                             int32_t num_requests,
                             const gbx_batch_options* options,
                             void* stream,
                             const gbx_allocator* mr,
                             gbx_batch** out);

/* Runs the batch on `stream` and waits for it; *out stays valid until the
 * next execute, rebind or destroy. */
GBX_API int gbx_batch_execute(gbx_batch* batch, void* stream, const gbx_batch_output** out);

/* Points the batch at new input buffers of the same schema and the same row
 * count per instance (tables, tuning and graph are kept). */
GBX_API int gbx_batch_rebind(gbx_batch* batch, const gbx_batch_instance* instances, int32_t num_instances);

/* The tuner's choice for each instance (mode and table slots) and its
 * estimated group count; arrays of num_instances entries, any may be NULL. */
GBX_API int gbx_batch_instance_plan(const gbx_batch* batch, int32_t* modes, int64_t* table_slots,
                                    int64_t* estimated_groups);

GBX_API int gbx_batch_last_stats(const gbx_batch* batch, gbx_batch_stats* out);
GBX_API void gbx_batch_destroy(gbx_batch* batch);

/* ---- served groupby -------------------------------------------------------
 * No counterpart in the reference (a libcudf service calls groupby::aggregate
 * per request on its own threads and streams).
 *
 * A server accepts groupby requests over device-resident columns as they
 * arrive and runs them with continuous batching: `workers` requests (or
 * merged batches) are on the GPU at once, each on its own stream, so their
 * kernels overlap; a request is admitted when a worker is free and the
 * device memory it may need fits the HBM budget beside the requests already
 * admitted (requests are considered in arrival order, and a later one that
 * fits may go ahead of one that does not); small requests of one schema that
 * are waiting together are merged into one batched launch (gbx_batch, one
 * shot).  Every result is the same as gbx_groupby_aggregate on that request
 * alone: same groups and dtypes, integer results bit-identical, floating
 * results within the stated summation bound (the accumulation order of
 * atomics is not fixed, as in the reference).
 *
 * gbx_server_submit copies the request's descriptors (the caller keeps the
 * column buffers alive until the request completes) and returns at once;
 * gbx_server_wait blocks until that request is done and hands over its
 * result (released with gbx_result_release).  Times are taken on the host's
 * steady clock, in seconds since the server was created. */
typedef struct gbx_server gbx_server;

typedef struct gbx_server_options {
  int32_t workers;              /* requests on the GPU at once (streams); 0: 4 */
  int32_t null_policy;          /* GBX_NULL_EXCLUDE / INCLUDE for every request */
  int64_t hbm_budget_bytes;     /* device memory admitted requests may hold; 0: 150 GB */
  int64_t batch_max_rows;       /* requests of at most this many rows may be merged (0: never) */
  int32_t batch_max_requests;   /* at most this many requests per merged launch; 0: 64 */
  int32_t large_in_flight;      /* large requests on the GPU at once; 0: 1 */
  int64_t large_rows;           /* a request of at least this many rows is large (it fills the GPU
                                   by itself and runs on a low-priority stream; smaller requests
                                   may pass a waiting large one); 0: 4M rows, < 0: none is large */
} gbx_server_options;

typedef struct gbx_server_timing {
  double submitted_s;      /* gbx_server_submit */
  double admitted_s;       /* given a worker and memory */
  double done_s;           /* result ready on the host side */
  int64_t reserved_bytes;  /* admission charge */
  int32_t batched;         /* number of requests in its launch (1: alone) */
  int32_t worker;
} gbx_server_timing;

typedef struct gbx_server_stats {
  int64_t submitted;
  int64_t completed;
  int64_t failed;
  int64_t batches;            /* merged launches */
  int64_t batched_requests;   /* requests served inside merged launches */
  int64_t peak_reserved_bytes;
  int64_t rows;               /* rows of completed requests */
  int32_t max_in_flight;
  int32_t workers;
  double busy_s;              /* time with at least one request on the GPU */
} gbx_server_stats;

GBX_API int gbx_server_create(const gbx_server_options* options, gbx_server** out);

/* Queues a request: `keys` and `requests` as for gbx_groupby_create /
 * gbx_groupby_aggregate.  Validation errors are returned here. */
GBX_API int gbx_server_submit(gbx_server* server, const gbx_table_view* keys, const gbx_request* requests,
                              int32_t num_requests, uint64_t* ticket);

/* Waits up to timeout_s seconds (< 0: no limit) for the request; returns
 * GBX_ERR_LOGIC with a message starting "timeout" if it is not done by then
 * (the ticket stays valid).  On completion *out receives the result (or the
 * request's error code is returned) and the ticket is retired. */
GBX_API int gbx_server_wait(gbx_server* server, uint64_t ticket, double timeout_s, gbx_result** out,
                            gbx_server_timing* timing);

GBX_API double gbx_server_now(const gbx_server* server);
GBX_API int gbx_server_last_stats(const gbx_server* server, gbx_server_stats* out);

/* Finishes the admitted requests, fails the waiting ones, and frees the server. */
GBX_API void gbx_server_destroy(gbx_server* server);

/* ---- distinct rows and a distinct-key hash join on the same tables --------
 * cudf::null_equality / nan_equality (types.hpp:143-154) and
 * duplicate_keep_option (stream_compaction.hpp:225-230). */
#define GBX_NULLS_EQUAL 0
#define GBX_NULLS_UNEQUAL 1
#define GBX_NANS_EQUAL 0   /* nan_equality::ALL_EQUAL */
#define GBX_NANS_UNEQUAL 1
typedef enum gbx_duplicate_keep {
  GBX_KEEP_ANY   = 0,
  GBX_KEEP_FIRST = 1,
  GBX_KEEP_LAST  = 2,
  GBX_KEEP_NONE  = 3
} gbx_duplicate_keep;

/* cudf::distinct_count(table_view, null_equality) (stream_compaction.hpp:422-424):
 * the number of distinct rows of `keys` (NaNs equal, -0.0 == +0.0; under
 * GBX_NULLS_UNEQUAL every row holding a null is distinct).  Synchronises
 * `stream`. */
GBX_API int gbx_distinct_count(const gbx_table_view* keys, int32_t nulls_equal, void* stream,
                               const gbx_allocator* mr, int64_t* out);

/* cudf::distinct_indices(table_view, keep, nulls_equal, nans_equal)
 * (stream_compaction.hpp:311-317): an INT32 column of the row indices kept,
 * one per distinct row (KEEP_ANY / FIRST / LAST: the first / first / last
 * row of each; KEEP_NONE: rows whose key occurs once), in no particular
 * order, allocated from `mr`.  Release it with gbx_column_release. */
GBX_API int gbx_distinct_indices(const gbx_table_view* keys, int32_t keep, int32_t nulls_equal, int32_t nans_equal,
                                 void* stream, const gbx_allocator* mr, gbx_column* out);

/* cudf::distinct_hash_join(build, probe, has_nulls, compare_nulls)
 * (join.hpp:494-533), the build side's keys distinct:
 *   join_kind 0 (inner_join): `build_indices` / `probe_indices` INT32 columns
 *     of the matching row pairs, in no particular order;
 *   join_kind 1 (left_join): `build_indices` holds, for every probe row, its
 *     build row or INT32_MIN (JoinNoneValue) and `probe_indices` is left
 *     empty.
 * Key columns must agree in count and type; dictionary keys are refused.
 * NaN keys match NaN keys.  Under GBX_NULLS_UNEQUAL a key holding a null
 * matches nothing.  A build key that occurs more than once answers its
 * first row.  Columns are allocated from `mr`. */
GBX_API int gbx_distinct_join(const gbx_table_view* build, const gbx_table_view* probe, int32_t compare_nulls,
                              int32_t join_kind, void* stream, const gbx_allocator* mr, gbx_column* build_indices,
                              gbx_column* probe_indices);

/* Hash joins (cudf::inner_join / left_join / full_join, join.hpp:107-190;
 * cudf::left_semi_join / left_anti_join, join.hpp:200-260).  `left` and
 * `right` have the same key columns (type, scale; STRUCT members alike):
 * fixed-width, STRING or STRUCT, not DICTIONARY32.  Returns INT32 gather maps
 * in no particular order (as the reference's): INNER the matching (left,
 * right) row pairs; LEFT every left row with each matching right row, or
 * GBX_JOIN_NONE; FULL the left join's pairs and then (GBX_JOIN_NONE, right
 * row) for every right row that matched nothing; LEFT_SEMI / LEFT_ANTI the
 * left rows with / without a match in `left_indices` (`right_indices` empty).
 * compare_nulls GBX_NULLS_EQUAL: nulls are equal, at every nesting level;
 * GBX_NULLS_UNEQUAL: a row holding a null anywhere in its key matches no
 * row.  NaNs are equal, -0.0 == +0.0.  Free both outputs with
 * gbx_column_release. */
typedef enum gbx_join_kind {
  GBX_JOIN_INNER     = 0,
  GBX_JOIN_LEFT      = 1,
  GBX_JOIN_FULL      = 2,
  GBX_JOIN_LEFT_SEMI = 3,
  GBX_JOIN_LEFT_ANTI = 4
} gbx_join_kind;
#define GBX_JOIN_NONE INT32_MIN /* cudf::JoinNoneValue */
GBX_API int gbx_hash_join(const gbx_table_view* left, const gbx_table_view* right, int32_t compare_nulls,
                          int32_t join_kind, void* stream, const gbx_allocator* mr, gbx_column* left_indices,
                          gbx_column* right_indices);

/* Frees a column returned by gbx_distinct_indices / gbx_distinct_join / gbx_hash_join with
 * the allocator that made it. */
GBX_API void gbx_column_release(gbx_column* col, const gbx_allocator* mr, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GBX_H */
