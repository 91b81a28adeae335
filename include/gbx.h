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

#define GBX_ABI_VERSION 1

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
  GBX_ERR_UNSUPPORTED = 4, /* valid in libcudf, but only on its sort-based path (not provided) */
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
  int32_t reserved0;
  const struct gbx_column_view* dict_keys;
} gbx_column_view;

typedef struct gbx_table_view {
  int32_t num_columns;
  int32_t reserved0;
  const gbx_column_view* columns;
} gbx_table_view;

/* One aggregation of a request (cudf::groupby_aggregation).  `ddof` is used by
 * VARIANCE/STD (make_variance_aggregation(ddof), aggregation.hpp:311-337).
 * COUNT's null_policy is encoded in the kind: COUNT_VALID (EXCLUDE) or
 * COUNT_ALL (INCLUDE), as make_count_aggregation does (aggregation.cpp:494-499). */
typedef struct gbx_aggregation {
  int32_t kind;
  int32_t ddof;
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
 * with the reference).  `keys_are_sorted` is accepted for API parity; the hash
 * path is used either way and group order is unspecified. */
GBX_API int gbx_groupby_create(const gbx_table_view* keys,
                       int32_t null_policy,
                       int32_t keys_are_sorted,
                       gbx_groupby** out);

/* cudf::groupby::groupby::aggregate (groupby.hpp:187-199, groupby.cu:197-221).
 * Validates requests (size mismatch and invalid type/aggregation combinations
 * fail with GBX_ERR_LOGIC, like CUDF_EXPECTS), runs the hash path on `stream`
 * and returns owning results allocated from `mr` (NULL: cudaMallocAsync).
 * Synchronises `stream` once, to learn the number of groups (the reference's
 * retrieve_all does the same).  On success *out must be freed with
 * gbx_result_release. */
GBX_API int gbx_groupby_aggregate(gbx_groupby* gb,
                          const gbx_request* requests,
                          int32_t num_requests,
                          void* stream,
                          const gbx_allocator* mr,
                          gbx_result** out);

/* Whether every request is computable by the hash path
 * (can_use_hash_groupby, hash/groupby.cu:635-651).  Returns 1/0, or -1 with
 * gbx_last_error() set on malformed input. */
GBX_API int gbx_can_use_hash_groupby(const gbx_request* requests, int32_t num_requests);

/* Output type of aggregation `kind` over a column of `type_id`
 * (cudf::detail::target_type, detail/aggregation/aggregation.hpp:1212-1335);
 * returns GBX_TYPE_EMPTY when the combination is invalid. */
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
  GBX_STRATEGY_WARP       = 4  /* per-warp private shared-memory tables, no atomics on the hot path */
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
  float init_ms;         /* table identity fill */
  float aggregate_ms;    /* the aggregation pass over the rows */
  float compact_ms;      /* occupied-slot compaction */
  float finalize_ms;     /* output keys/results + null counts */
  float total_ms;        /* first to last event of the call */
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
 * GBX_NOALLOC_SCRATCH_BYTES inside libgbx (every GPU that loads the library
 * holds it until the process exits), and the caller passes every output
 * buffer.
 *
 * Limits: at most GBX_NOALLOC_MAX_GROUPS groups (more is rejected with
 * GBX_ERR_LOGIC after the aggregation pass, outputs untouched), and the
 * aggregations' per-group state must fit the array (else GBX_ERR_LOGIC).
 *
 * Outputs: `out_keys` has one gbx_column per key column and `out_results` one
 * per aggregation of every request, in request order.  The caller sets each
 * column's `data` (room for `capacity` rows of the output type, see
 * gbx_target_type) and `null_mask` (room for `capacity` bits in 32-bit words;
 * required where the output can hold nulls, ignored otherwise); the call
 * fills each `view` and `*num_groups`.
 *
 * Every call shares the one array: calls whose work overlaps on the GPU (on
 * different streams or threads) race and corrupt each other's results, so
 * serialise them.  The array keeps the last call's contents; each call clears
 * what must start at zero itself.  The first call on a device looks up the
 * array's device address (once per device); it synchronises `stream` twice,
 * as gbx_groupby_aggregate does. */
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

#ifdef __cplusplus
}
#endif

#endif /* GBX_H */
