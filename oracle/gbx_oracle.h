/*
 * gbx_oracle.h -- CPU oracle for the hash groupby-aggregation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of libcudf 24.10's
 * hash groupby semantics used as the parity checker (tests, the smoke check and
 * the CPU baseline of the benchmark).  Nothing in the product (libgbx) links,
 * loads or calls it.
 *
 * Inputs use the same POD descriptors as the product's C ABI (include/gbx.h),
 * but every data / null_mask pointer here is HOST memory.
 */
#ifndef GBX_ORACLE_H
#define GBX_ORACLE_H

#include "../include/gbx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One oracle output column: host buffers owned by the result.
 * `valid` is one byte per row (1 = valid); it is NULL when the column has no
 * null mask in the reference's output (every row valid). */
typedef struct gbo_column {
  int32_t type_id;
  int32_t scale;
  int64_t size;
  void* data;
  uint8_t* valid;
  /* DICTIONARY32 output keys: data holds int32 indices into the input's keys;
   * STRING output keys: data holds the characters and str_offsets the
   * size + 1 offsets into them */
  int64_t* str_offsets;
} gbo_column;

typedef struct gbo_result {
  int64_t num_groups;
  int32_t num_key_columns;
  int32_t num_requests;
  gbo_column* keys;
  int32_t* num_results; /* per request */
  gbo_column** results; /* per request, per aggregation */
} gbo_result;

/* Runs the groupby on host data with `threads` worker threads (1 = the plain
 * restatement; >1 hash-partitions the groups across threads).  Returns GBX_OK
 * or a gbx_status code; the message is available from gbo_last_error(). */
int gbo_groupby(const gbx_table_view* keys,
                int32_t null_policy,
                const gbx_request* requests,
                int32_t num_requests,
                int32_t threads,
                gbo_result** out);

void gbo_result_free(gbo_result* r);
const char* gbo_last_error(void);
int32_t gbo_target_type(int32_t type_id, int32_t kind);

#ifdef __cplusplus
}
#endif
#endif
