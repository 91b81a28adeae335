/*
 * gbx_oracle.c -- CPU oracle for libcudf's hash groupby-aggregation path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker and the CPU baseline); the
 * product never links or calls this file.
 *
 * It restates, in plain C, the algorithm of libcudf 24.10's hash groupby:
 *   - rows whose key has a null are skipped under null_policy EXCLUDE
 *     (bitmask_and of the key masks: cpp/src/groupby/hash/groupby.cu:482-485,
 *      cpp/src/groupby/hash/groupby_kernels.cuh:98-105);
 *   - a set of representative ROW INDICES with linear probing, load 0.5,
 *     sized by rows (hash/groupby.cu:571-580), hashed by a row hasher that
 *     normalises -0.0/+0.0 and NaNs (hashing/detail/hash_functions.cuh:41-47)
 *     and compared with nulls-equal, NaN-equal element equality
 *     (table/experimental/row_operators.cuh:1285-1312, 1429-1447);
 *   - each row then updates one accumulator per flattened aggregation with
 *     null values skipped (detail/aggregation/aggregation.cuh:116-491, 558-573);
 *     MEAN/VAR/STD are flattened into SUM + COUNT_VALID (hash/groupby.cu:113-181);
 *   - VAR is a second pass over all rows: sum((x - sum/n)^2) / (n - ddof), null
 *     when n - ddof <= 0 (hash/multi_pass_kernels.cuh:74-111); STD = sqrt(VAR)
 *     (hash/groupby.cu:339-348); MEAN = SUM / COUNT (hash/groupby.cu:287-306);
 *   - result types follow cudf::detail::target_type
 *     (detail/aggregation/aggregation.hpp:1212-1335); a result is nullable iff
 *     the value column has nulls, COUNT never, VAR/STD always
 *     (hash/groupby.cu:424-454).
 *
 * Arithmetic: integer SUM/PRODUCT/SUM_OF_SQUARES wrap in 64-bit two's
 * complement (the reference's atomicAdd on unsigned long long,
 * detail/utilities/device_atomics.cuh:195-205).  Floating sums and the VAR
 * second pass accumulate in long double (at least FP64), so the oracle is at
 * least as accurate as an FP64 reference.
 *
 * MIN/MAX of floating values containing NaN depend on atomic order in the
 * reference (a CAS loop with `a < b ? a : b`, fixed_point/temporary.hpp:63-72);
 * the oracle fixes one of those orders: NaN values are ignored unless every
 * valid value of the group is NaN, in which case the result is NaN.
 * ARGMIN/ARGMAX ties resolve to the lowest row index, NaN handled the same way.
 *
 * The kinds libcudf computes on its sort path are restated from there:
 * M2 = sum((x - mean)^2) with MEAN's mask (groupby/sort/group_m2.cu);
 * MEDIAN / QUANTILE select from each group's valid values sorted with NaN
 * last, -0.0 == +0.0 and ties in row order (groupby/sort/sort_helper.cu:
 * 251-272, group_quantiles.cu, quantiles/quantiles_util.hpp:39-190), in
 * double arithmetic in the reference's order; NUNIQUE counts distinct valid
 * values, NaNs equal, and the nulls as one value under INCLUDE
 * (groupby/sort/group_nunique.cu:63-72); NTH_ELEMENT takes the n-th row of a
 * group in row order, null values dropped first under EXCLUDE, null when out
 * of range, without a mask when no output is null
 * (groupby/sort/group_nth_element.cu).
 *
 * Groups come out in first-occurrence order; callers sort by key to compare.
 */
#define _GNU_SOURCE
#include "gbx_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[512];

static int set_err(int code, const char* fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

const char* gbo_last_error(void) { return g_err; }

/* ---------------------------------------------------------------- types --- */

enum { CAT_NONE = 0, CAT_SIGNED, CAT_UNSIGNED, CAT_FLOAT, CAT_BOOL };

static int type_width(int32_t t)
{
  switch (t) {
    case GBX_TYPE_INT8:
    case GBX_TYPE_UINT8:
    case GBX_TYPE_BOOL8: return 1;
    case GBX_TYPE_INT16:
    case GBX_TYPE_UINT16: return 2;
    case GBX_TYPE_INT32:
    case GBX_TYPE_UINT32:
    case GBX_TYPE_FLOAT32:
    case GBX_TYPE_TIMESTAMP_DAYS:
    case GBX_TYPE_DURATION_DAYS:
    case GBX_TYPE_DECIMAL32:
    case GBX_TYPE_DICTIONARY32: return 4;
    case GBX_TYPE_INT64:
    case GBX_TYPE_UINT64:
    case GBX_TYPE_FLOAT64:
    case GBX_TYPE_TIMESTAMP_SECONDS:
    case GBX_TYPE_TIMESTAMP_MILLISECONDS:
    case GBX_TYPE_TIMESTAMP_MICROSECONDS:
    case GBX_TYPE_TIMESTAMP_NANOSECONDS:
    case GBX_TYPE_DURATION_SECONDS:
    case GBX_TYPE_DURATION_MILLISECONDS:
    case GBX_TYPE_DURATION_MICROSECONDS:
    case GBX_TYPE_DURATION_NANOSECONDS:
    case GBX_TYPE_DECIMAL64: return 8;
    default: return 0;
  }
}

static int type_cat(int32_t t)
{
  switch (t) {
    case GBX_TYPE_INT8:
    case GBX_TYPE_INT16:
    case GBX_TYPE_INT32:
    case GBX_TYPE_INT64:
    case GBX_TYPE_TIMESTAMP_DAYS:
    case GBX_TYPE_TIMESTAMP_SECONDS:
    case GBX_TYPE_TIMESTAMP_MILLISECONDS:
    case GBX_TYPE_TIMESTAMP_MICROSECONDS:
    case GBX_TYPE_TIMESTAMP_NANOSECONDS:
    case GBX_TYPE_DURATION_DAYS:
    case GBX_TYPE_DURATION_SECONDS:
    case GBX_TYPE_DURATION_MILLISECONDS:
    case GBX_TYPE_DURATION_MICROSECONDS:
    case GBX_TYPE_DURATION_NANOSECONDS:
    case GBX_TYPE_DECIMAL32:
    case GBX_TYPE_DECIMAL64: return CAT_SIGNED;
    case GBX_TYPE_UINT8:
    case GBX_TYPE_UINT16:
    case GBX_TYPE_UINT32:
    case GBX_TYPE_UINT64: return CAT_UNSIGNED;
    case GBX_TYPE_BOOL8: return CAT_BOOL;
    case GBX_TYPE_FLOAT32:
    case GBX_TYPE_FLOAT64: return CAT_FLOAT;
    default: return CAT_NONE;
  }
}

static int is_integral(int32_t t)
{
  return (t >= GBX_TYPE_INT8 && t <= GBX_TYPE_UINT64) || t == GBX_TYPE_BOOL8;
}
static int is_floating(int32_t t) { return t == GBX_TYPE_FLOAT32 || t == GBX_TYPE_FLOAT64; }
static int is_duration(int32_t t)
{
  return t >= GBX_TYPE_DURATION_DAYS && t <= GBX_TYPE_DURATION_NANOSECONDS;
}
static int is_decimal(int32_t t) { return t == GBX_TYPE_DECIMAL32 || t == GBX_TYPE_DECIMAL64; }
static int is_fixed_width(int32_t t) { return type_width(t) > 0 && t != GBX_TYPE_DICTIONARY32; }

/* cudf::detail::target_type restated (detail/aggregation/aggregation.hpp:1212-1367)
 * for the hash path's kinds (hash/groupby.cu:73-84, 635-651) and the sort
 * path's M2, MEDIAN, QUANTILE, NUNIQUE and NTH_ELEMENT. */
int32_t gbo_target_type(int32_t t, int32_t kind)
{
  if (!is_fixed_width(t)) return GBX_TYPE_EMPTY;
  switch (kind) {
    case GBX_AGG_SUM:
      if (is_integral(t)) return GBX_TYPE_INT64;
      if (is_floating(t) || is_duration(t) || is_decimal(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_PRODUCT:
    case GBX_AGG_SUM_OF_SQUARES:
      if (is_integral(t)) return GBX_TYPE_INT64;
      if (is_floating(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_MIN:
    case GBX_AGG_MAX: return t;
    case GBX_AGG_COUNT_VALID:
    case GBX_AGG_COUNT_ALL: return GBX_TYPE_INT32;
    case GBX_AGG_ARGMIN:
    case GBX_AGG_ARGMAX: return GBX_TYPE_INT32;
    case GBX_AGG_MEAN:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      if (is_duration(t) || is_decimal(t)) return t;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_VARIANCE:
    case GBX_AGG_STD:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      return GBX_TYPE_EMPTY;
    /* sort-path kinds (aggregation.hpp:1318-1367): M2 / MEDIAN / QUANTILE
     * are double over arithmetic values, NUNIQUE a size_type count,
     * NTH_ELEMENT the value's own type */
    case GBX_AGG_M2:
    case GBX_AGG_MEDIAN:
    case GBX_AGG_QUANTILE:
      if (is_integral(t) || is_floating(t)) return GBX_TYPE_FLOAT64;
      return GBX_TYPE_EMPTY;
    case GBX_AGG_NUNIQUE: return GBX_TYPE_INT32;
    case GBX_AGG_NTH_ELEMENT: return t;
    default: return GBX_TYPE_EMPTY;
  }
}

/* --------------------------------------------------------- element access --- */

typedef struct {
  int32_t type_id; /* physical type of the value (dictionary resolved) */
  int64_t i;       /* signed / bool */
  uint64_t u;      /* unsigned */
  long double f;   /* floating */
} scalar;

static int bit_valid(const uint32_t* mask, int64_t i)
{
  return mask == NULL || ((mask[i >> 5] >> (i & 31)) & 1u);
}

static int col_valid(const gbx_column_view* c, int64_t row)
{
  return bit_valid(c->null_mask, row + c->offset);
}

static int64_t read_signed(const void* data, int w, int64_t i)
{
  switch (w) {
    case 1: return ((const int8_t*)data)[i];
    case 2: return ((const int16_t*)data)[i];
    case 4: return ((const int32_t*)data)[i];
    default: return ((const int64_t*)data)[i];
  }
}

static uint64_t read_unsigned(const void* data, int w, int64_t i)
{
  switch (w) {
    case 1: return ((const uint8_t*)data)[i];
    case 2: return ((const uint16_t*)data)[i];
    case 4: return ((const uint32_t*)data)[i];
    default: return ((const uint64_t*)data)[i];
  }
}

/* Value of a fixed-width column at `row` (view offset applied). */
static scalar read_fixed(const gbx_column_view* c, int64_t row)
{
  scalar s;
  memset(&s, 0, sizeof(s));
  s.type_id   = c->type_id;
  int64_t idx = row + c->offset;
  int w       = type_width(c->type_id);
  switch (type_cat(c->type_id)) {
    case CAT_SIGNED: s.i = read_signed(c->data, w, idx); break;
    case CAT_UNSIGNED: s.u = read_unsigned(c->data, w, idx); break;
    case CAT_BOOL: s.i = ((const uint8_t*)c->data)[idx] != 0; break;
    case CAT_FLOAT:
      s.f = (c->type_id == GBX_TYPE_FLOAT32) ? (long double)((const float*)c->data)[idx]
                                             : (long double)((const double*)c->data)[idx];
      break;
  }
  return s;
}

static int64_t dict_index(const gbx_column_view* c, int64_t row)
{
  int32_t it  = c->index_type_id ? c->index_type_id : GBX_TYPE_INT32;
  int64_t idx = row + c->offset;
  if (type_cat(it) == CAT_UNSIGNED) return (int64_t)read_unsigned(c->data, type_width(it), idx);
  return read_signed(c->data, type_width(it), idx);
}

/* Value of a value column (dictionary resolved through its keys, as
 * update_target_element<dictionary32,...> does, aggregation.cuh:324-348). */
static scalar read_value(const gbx_column_view* c, int64_t row)
{
  if (c->type_id == GBX_TYPE_DICTIONARY32) {
    int64_t k = dict_index(c, row);
    return read_fixed(c->dict_keys, k);
  }
  return read_fixed(c, row);
}

static int32_t value_type(const gbx_column_view* c)
{
  return c->type_id == GBX_TYPE_DICTIONARY32 ? c->dict_keys->type_id : c->type_id;
}

/* ------------------------------------------------------------- row hash --- */

static uint64_t fmix64(uint64_t k)
{
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

/* STRING element `row`: its bytes and length (the offsets child in dict_keys). */
static const unsigned char* str_at(const gbx_column_view* c, int64_t row, int64_t* len)
{
  const gbx_column_view* o = c->dict_keys;
  int w                    = type_width(o->type_id);
  int64_t i                = row + c->offset + o->offset;
  int64_t a                = w == 4 ? ((const int32_t*)o->data)[i] : ((const int64_t*)o->data)[i];
  int64_t b                = w == 4 ? ((const int32_t*)o->data)[i + 1] : ((const int64_t*)o->data)[i + 1];
  *len                     = b - a;
  return (const unsigned char*)c->data + a;
}

/* Normalised bits of a key element: -0.0 -> +0.0 and every NaN -> one NaN,
 * as normalize_nans_and_zeros does before hashing (hash_functions.cuh:41-47). */
static uint64_t key_bits(const gbx_column_view* c, int64_t row)
{
  if (c->type_id == GBX_TYPE_DICTIONARY32) return (uint64_t)dict_index(c, row);
  if (c->type_id == GBX_TYPE_STRING) {
    /* a hash of the bytes (equality compares the bytes themselves) */
    int64_t len;
    const unsigned char* s = str_at(c, row, &len);
    uint64_t h             = 1469598103934665603ULL ^ (uint64_t)len;
    for (int64_t j = 0; j < len; ++j) h = (h ^ s[j]) * 1099511628211ULL;
    return h;
  }
  scalar s = read_fixed(c, row);
  switch (type_cat(c->type_id)) {
    case CAT_SIGNED:
    case CAT_BOOL: return (uint64_t)s.i;
    case CAT_UNSIGNED: return s.u;
    case CAT_FLOAT: {
      double d = (double)s.f;
      if (isnan(d)) return 0x7ff8000000000000ULL;
      if (d == 0.0) return 0;
      uint64_t b;
      memcpy(&b, &d, 8);
      return b;
    }
  }
  return 0;
}

typedef struct {
  const gbx_table_view* keys;
  int check_nulls;
} row_ops;

static uint64_t row_hash(const row_ops* ops, int64_t row)
{
  uint64_t h = 0;
  for (int c = 0; c < ops->keys->num_columns; ++c) {
    const gbx_column_view* col = &ops->keys->columns[c];
    uint64_t e = (ops->check_nulls && !col_valid(col, row)) ? 0xffffffffffffffffULL
                                                            : fmix64(key_bits(col, row) + 0x9e37ULL);
    h = fmix64(h ^ (e + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2)));
  }
  return h;
}

/* Nulls compare equal; NaN == NaN; -0.0 == +0.0 (row_operators.cuh:1285-1312, 1429-1447). */
static int row_equal(const row_ops* ops, int64_t a, int64_t b)
{
  for (int c = 0; c < ops->keys->num_columns; ++c) {
    const gbx_column_view* col = &ops->keys->columns[c];
    if (ops->check_nulls) {
      int va = col_valid(col, a), vb = col_valid(col, b);
      if (!va && !vb) continue;
      if (va != vb) return 0;
    }
    if (col->type_id == GBX_TYPE_STRING) {
      int64_t la, lb;
      const unsigned char* sa = str_at(col, a, &la);
      const unsigned char* sb = str_at(col, b, &lb);
      if (la != lb || (la > 0 && memcmp(sa, sb, (size_t)la) != 0)) return 0;
      continue;
    }
    if (key_bits(col, a) != key_bits(col, b)) return 0;
  }
  return 1;
}

/* ------------------------------------------------------- flattened aggs --- */

/* One accumulator per (request, simple aggregation kind); MEAN/VAR/STD use
 * the SUM and COUNT_VALID of their request (hash/groupby.cu:113-181, 351-383). */
typedef struct {
  long double fsum;    /* floating SUM (and float MEAN/VAR input) */
  int64_t isum;        /* integral/duration/decimal SUM, wraps */
  long double fprod;
  int64_t iprod;
  long double fsq;
  int64_t isq;
  int64_t count_valid;
  int64_t count_all;
  scalar minv, maxv;   /* over non-NaN values */
  int has_min;         /* some non-NaN valid value seen */
  int saw_nan;         /* some NaN valid value seen */
  int64_t argmin, argmax;
  long double m2;      /* VAR second pass */
} accum;

static int scalar_less(const scalar* a, const scalar* b)
{
  switch (type_cat(a->type_id)) {
    case CAT_SIGNED:
    case CAT_BOOL: return a->i < b->i;
    case CAT_UNSIGNED: return a->u < b->u;
    case CAT_FLOAT: return a->f < b->f;
  }
  return 0;
}

static int scalar_isnan(const scalar* a)
{
  return type_cat(a->type_id) == CAT_FLOAT && isnan((double)a->f);
}

static long double scalar_as_ld(const scalar* a)
{
  switch (type_cat(a->type_id)) {
    case CAT_SIGNED:
    case CAT_BOOL: return (long double)a->i;
    case CAT_UNSIGNED: return (long double)a->u;
    default: return a->f;
  }
}

static int64_t scalar_as_i64(const scalar* a)
{
  switch (type_cat(a->type_id)) {
    case CAT_SIGNED:
    case CAT_BOOL: return a->i;
    case CAT_UNSIGNED: return (int64_t)a->u;
    default: return (int64_t)a->f;
  }
}

static void accum_init(accum* a)
{
  memset(a, 0, sizeof(*a));
  a->fprod  = 1.0L;
  a->iprod  = 1;
  a->argmin = -1;
  a->argmax = -1;
}

static void accum_update(accum* a, const gbx_column_view* col, int64_t row)
{
  a->count_all++;
  int valid = col_valid(col, row);
  if (!valid) return;
  a->count_valid++;
  scalar v = read_value(col, row);
  if (type_cat(v.type_id) == CAT_FLOAT) {
    a->fsum += v.f;
    a->fprod *= v.f;
    a->fsq += v.f * v.f;
  } else {
    int64_t x = scalar_as_i64(&v);
    a->isum   = (int64_t)((uint64_t)a->isum + (uint64_t)x);
    a->iprod  = (int64_t)((uint64_t)a->iprod * (uint64_t)x);
    a->isq    = (int64_t)((uint64_t)a->isq + (uint64_t)x * (uint64_t)x);
  }
  if (scalar_isnan(&v)) {
    if (!a->saw_nan && !a->has_min) { a->argmin = row; a->argmax = row; }
    a->saw_nan = 1;
    return;
  }
  if (!a->has_min) {
    a->minv = v;
    a->maxv = v;
    a->argmin = row;
    a->argmax = row;
    a->has_min = 1;
    return;
  }
  if (scalar_less(&v, &a->minv)) { a->minv = v; a->argmin = row; }
  if (scalar_less(&a->maxv, &v)) { a->maxv = v; a->argmax = row; }
}

/* ----------------------------------------------------------- output cols --- */

static void* xcalloc(size_t n, size_t sz)
{
  void* p = calloc(n ? n : 1, sz ? sz : 1);
  return p;
}

static void store_scalar(void* data, int32_t t, int64_t i, const scalar* s)
{
  int w = type_width(t);
  switch (type_cat(t)) {
    case CAT_SIGNED:
    case CAT_BOOL:
      switch (w) {
        case 1: ((int8_t*)data)[i] = (int8_t)s->i; break;
        case 2: ((int16_t*)data)[i] = (int16_t)s->i; break;
        case 4: ((int32_t*)data)[i] = (int32_t)s->i; break;
        default: ((int64_t*)data)[i] = s->i; break;
      }
      break;
    case CAT_UNSIGNED:
      switch (w) {
        case 1: ((uint8_t*)data)[i] = (uint8_t)s->u; break;
        case 2: ((uint16_t*)data)[i] = (uint16_t)s->u; break;
        case 4: ((uint32_t*)data)[i] = (uint32_t)s->u; break;
        default: ((uint64_t*)data)[i] = s->u; break;
      }
      break;
    case CAT_FLOAT:
      if (t == GBX_TYPE_FLOAT32) ((float*)data)[i] = (float)s->f;
      else ((double*)data)[i] = (double)s->f;
      break;
  }
}

static void store_i64(void* data, int32_t t, int64_t i, int64_t v)
{
  scalar s;
  memset(&s, 0, sizeof(s));
  s.type_id = t;
  s.i       = v;
  s.u       = (uint64_t)v;
  store_scalar(data, t, i, &s);
}

/* ---------------------------------------------------------- the groupby --- */

typedef struct {
  /* inputs */
  const gbx_table_view* keys;
  int32_t null_policy;
  const gbx_request* requests;
  int32_t num_requests;
  int64_t num_rows;
  int skip_null_keys;
  int check_nulls;
  int32_t part, nparts;
  /* outputs */
  int64_t num_groups;
  int64_t* rep_row;   /* representative row per group */
  int64_t* row_gid;   /* each row's group in this worker (-1: another worker's, or skipped) */
  accum** acc;        /* per request: num_groups accumulators */
  int status;
} worker;

static int row_key_valid(const gbx_table_view* keys, int64_t row)
{
  for (int c = 0; c < keys->num_columns; ++c)
    if (!col_valid(&keys->columns[c], row)) return 0;
  return 1;
}

static void* run_worker(void* arg)
{
  worker* w     = (worker*)arg;
  row_ops ops   = {w->keys, w->check_nulls};
  int64_t n     = w->num_rows;
  /* static_set capacity: rows / 0.5 (hash/groupby.cu:571-575), power of two here */
  int64_t cap = 2;
  while (cap < 2 * (n / (w->nparts > 0 ? w->nparts : 1) + 1)) cap <<= 1;
  int64_t* slots  = (int64_t*)malloc((size_t)cap * sizeof(int64_t));
  int64_t* gid_of = (int64_t*)malloc((size_t)cap * sizeof(int64_t));
  int64_t* row_gid = (int64_t*)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
  if (!slots || !gid_of || !row_gid) {
    w->status = GBX_ERR_ALLOC;
    free(slots); free(gid_of); free(row_gid);
    return NULL;
  }
  for (int64_t i = 0; i < cap; ++i) slots[i] = -1; /* empty_key sentinel, cuco_helpers.hpp:27 */
  int64_t ng = 0, rep_cap = 1024;
  int64_t* rep = (int64_t*)malloc((size_t)rep_cap * sizeof(int64_t));

  /* pass 1: insert_and_find per row (groupby_kernels.cuh:98-105) */
  for (int64_t r = 0; r < n; ++r) {
    row_gid[r] = -1;
    if (w->skip_null_keys && !row_key_valid(w->keys, r)) continue;
    uint64_t h = row_hash(&ops, r);
    if (w->nparts > 1 && (int32_t)((h >> 40) % (uint64_t)w->nparts) != w->part) continue;
    int64_t s = (int64_t)(h & (uint64_t)(cap - 1));
    for (;;) {
      if (slots[s] < 0) {
        slots[s]  = r;
        gid_of[s] = ng;
        if (ng == rep_cap) {
          rep_cap *= 2;
          rep = (int64_t*)realloc(rep, (size_t)rep_cap * sizeof(int64_t));
        }
        rep[ng++] = r;
        row_gid[r] = gid_of[s];
        break;
      }
      if (row_equal(&ops, slots[s], r)) {
        row_gid[r] = gid_of[s];
        break;
      }
      s = (s + 1) & (cap - 1);
    }
  }
  free(slots);
  free(gid_of);

  /* single-pass aggregations: one accumulator set per request */
  w->acc = (accum**)xcalloc((size_t)w->num_requests, sizeof(accum*));
  for (int q = 0; q < w->num_requests; ++q) {
    accum* a = (accum*)xcalloc((size_t)ng, sizeof(accum));
    for (int64_t g = 0; g < ng; ++g) accum_init(&a[g]);
    const gbx_column_view* col = &w->requests[q].values;
    for (int64_t r = 0; r < n; ++r)
      if (row_gid[r] >= 0) accum_update(&a[row_gid[r]], col, r);
    /* VAR/STD second pass around sum/count (multi_pass_kernels.cuh:74-111) */
    int need_var = 0;
    for (int k = 0; k < w->requests[q].num_aggregations; ++k) {
      int32_t kind = w->requests[q].aggregations[k].kind;
      if (kind == GBX_AGG_VARIANCE || kind == GBX_AGG_STD || kind == GBX_AGG_M2) need_var = 1;
    }
    if (need_var) {
      for (int64_t r = 0; r < n; ++r) {
        int64_t g = row_gid[r];
        if (g < 0 || !col_valid(col, r)) continue;
        accum* ag = &a[g];
        if (ag->count_valid == 0) continue;
        scalar v     = read_value(col, r);
        long double x = scalar_as_ld(&v);
        long double sum = (type_cat(v.type_id) == CAT_FLOAT) ? ag->fsum : (long double)ag->isum;
        long double mean = sum / (long double)ag->count_valid;
        ag->m2 += (x - mean) * (x - mean);
      }
    }
    w->acc[q] = a;
  }
  w->row_gid    = row_gid;
  w->num_groups = ng;
  w->rep_row    = rep;
  w->status     = GBX_OK;
  return NULL;
}

static int validate(const gbx_table_view* keys, const gbx_request* reqs, int32_t nreq)
{
  if (!keys || keys->num_columns <= 0) return set_err(GBX_ERR_LOGIC, "keys table is empty");
  int64_t n = keys->columns[0].size;
  for (int c = 0; c < keys->num_columns; ++c) {
    const gbx_column_view* k = &keys->columns[c];
    if (k->size != n) return set_err(GBX_ERR_LOGIC, "key columns differ in size");
    if (k->type_id == GBX_TYPE_DICTIONARY32) {
      if (!k->dict_keys) return set_err(GBX_ERR_LOGIC, "dictionary key column without keys");
    } else if (k->type_id == GBX_TYPE_STRING) {
      if (!k->dict_keys) return set_err(GBX_ERR_LOGIC, "STRING key column without offsets");
    } else if (!is_fixed_width(k->type_id)) {
      return set_err(GBX_ERR_UNSUPPORTED, "key type %d not supported", k->type_id);
    }
  }
  for (int q = 0; q < nreq; ++q) {
    const gbx_request* r = &reqs[q];
    if (r->values.size != n)
      return set_err(GBX_ERR_LOGIC, "Size mismatch between request values and groupby keys.");
    int32_t vt = value_type(&r->values);
    for (int k = 0; k < r->num_aggregations; ++k) {
      if (gbo_target_type(vt, r->aggregations[k].kind) == GBX_TYPE_EMPTY)
        return set_err(GBX_ERR_LOGIC, "Invalid type/aggregation combination.");
      if (r->aggregations[k].kind == GBX_AGG_QUANTILE &&
          (r->aggregations[k].num_quantiles < 0 ||
           (r->aggregations[k].num_quantiles > 0 && r->aggregations[k].quantiles == NULL)))
        return set_err(GBX_ERR_LOGIC, "invalid quantile array");
    }
  }
  return GBX_OK;
}

static void finalize_column(gbo_column* out,
                            const gbx_request* req,
                            const gbx_aggregation* agg,
                            int64_t ng,
                            accum** per_group,
                            const int64_t* rep_row)
{
  (void)rep_row;
  const gbx_column_view* col = &req->values;
  int32_t vt                 = value_type(col);
  int32_t tt                 = gbo_target_type(vt, agg->kind);
  int has_nulls = 0;
  if (col->null_mask) {
    for (int64_t r = 0; r < col->size && !has_nulls; ++r) has_nulls = !col_valid(col, r);
  }
  int nullable = (agg->kind == GBX_AGG_COUNT_VALID || agg->kind == GBX_AGG_COUNT_ALL)
                   ? 0
                   : (has_nulls || agg->kind == GBX_AGG_VARIANCE || agg->kind == GBX_AGG_STD);
  out->type_id = tt;
  out->scale   = is_decimal(tt) ? ((col->type_id == GBX_TYPE_DICTIONARY32) ? col->dict_keys->scale
                                                                             : col->scale)
                                : 0;
  out->size    = ng;
  out->data    = xcalloc((size_t)ng, (size_t)type_width(tt));
  out->valid   = nullable ? (uint8_t*)xcalloc((size_t)ng, 1) : NULL;
  int fl       = is_floating(vt);
  for (int64_t g = 0; g < ng; ++g) {
    accum* a  = per_group[g];
    int valid = a->count_valid > 0;
    switch (agg->kind) {
      case GBX_AGG_SUM:
        if (fl) {
          scalar s = {tt, 0, 0, a->fsum};
          store_scalar(out->data, tt, g, &s);
        } else store_i64(out->data, tt, g, a->isum);
        break;
      case GBX_AGG_PRODUCT:
        if (fl) {
          scalar s = {tt, 0, 0, a->fprod};
          store_scalar(out->data, tt, g, &s);
        } else store_i64(out->data, tt, g, a->iprod);
        break;
      case GBX_AGG_SUM_OF_SQUARES:
        if (fl) {
          scalar s = {tt, 0, 0, a->fsq};
          store_scalar(out->data, tt, g, &s);
        } else store_i64(out->data, tt, g, a->isq);
        break;
      case GBX_AGG_MIN:
      case GBX_AGG_MAX: {
        if (!valid) break;
        scalar s;
        if (a->has_min) s = (agg->kind == GBX_AGG_MIN) ? a->minv : a->maxv;
        else {
          memset(&s, 0, sizeof(s));
          s.type_id = vt;
          s.f       = (long double)NAN;
        }
        s.type_id = tt;
        store_scalar(out->data, tt, g, &s);
        break;
      }
      case GBX_AGG_COUNT_VALID: ((int32_t*)out->data)[g] = (int32_t)a->count_valid; break;
      case GBX_AGG_COUNT_ALL: ((int32_t*)out->data)[g] = (int32_t)a->count_all; break;
      case GBX_AGG_ARGMIN: ((int32_t*)out->data)[g] = valid ? (int32_t)a->argmin : -1; break;
      case GBX_AGG_ARGMAX: ((int32_t*)out->data)[g] = valid ? (int32_t)a->argmax : -1; break;
      case GBX_AGG_MEAN:
        if (!valid) break;
        if (tt == GBX_TYPE_FLOAT64) {
          long double sum = fl ? a->fsum : (long double)a->isum;
          ((double*)out->data)[g] = (double)(sum / (long double)a->count_valid);
        } else {
          /* durations / decimals: integer division of the rep (binaryop DIV) */
          store_i64(out->data, tt, g, a->isum / a->count_valid);
        }
        break;
      case GBX_AGG_VARIANCE:
      case GBX_AGG_STD: {
        int64_t n  = a->count_valid;
        int64_t dd = agg->ddof;
        if (n == 0 || n - dd <= 0) {
          valid = 0;
          break;
        }
        long double var = a->m2 / (long double)(n - dd);
        ((double*)out->data)[g] =
          (agg->kind == GBX_AGG_STD) ? (double)sqrtl(var) : (double)var;
        valid = 1;
        break;
      }
      case GBX_AGG_M2:
        /* sum((x - mean)^2) over the valid values, mean = SUM / COUNT_VALID,
         * with MEAN's mask: nullable iff the values have nulls, null where
         * the group has no valid value (group_m2.cu:37-52, 97-101) */
        if (valid) ((double*)out->data)[g] = (double)a->m2;
        break;
    }
    if (out->valid) out->valid[g] = (uint8_t)valid;
  }
}

/* ------------------------------------------------ sort-path kinds --- */

static int is_sorted_kind(int32_t k)
{
  return k == GBX_AGG_MEDIAN || k == GBX_AGG_QUANTILE || k == GBX_AGG_NUNIQUE || k == GBX_AGG_NTH_ELEMENT;
}

typedef struct {
  scalar v;
  int64_t row;
} sorted_value;

/* The reference's value order: NaN after every number and NaNs equal;
 * -0.0 == +0.0 (the `<` comparisons). */
static int value_cmp(const scalar* a, const scalar* b)
{
  if (type_cat(a->type_id) == CAT_FLOAT) {
    int na = isnan((double)a->f), nb = isnan((double)b->f);
    if (na || nb) return na - nb;
  }
  if (scalar_less(a, b)) return -1;
  if (scalar_less(b, a)) return 1;
  return 0;
}

/* a stable sort by value: ties in row order */
static int sorted_value_cmp(const void* x, const void* y)
{
  const sorted_value* a = (const sorted_value*)x;
  const sorted_value* b = (const sorted_value*)y;
  int c                 = value_cmp(&a->v, &b->v);
  if (c) return c;
  return (a->row > b->row) - (a->row < b->row);
}

/* convert_to_floating<double> (quantiles_util.hpp) */
static double value_as_double(const scalar* a)
{
  switch (type_cat(a->type_id)) {
    case CAT_SIGNED:
    case CAT_BOOL: return (double)a->i;
    case CAT_UNSIGNED: return (double)a->u;
    default: return (double)a->f;
  }
}

/* quantile_index and select_quantile_data (quantiles_util.hpp:92-190) over
 * `count` sorted values, in double arithmetic in the reference's order. */
static double select_quantile(const sorted_value* v, int64_t count, double q, int32_t interp)
{
  q               = q < 0.0 ? 0.0 : (q > 1.0 ? 1.0 : q);
  double val      = q * (double)(count - 1);
  int64_t lo      = (int64_t)floor(val);
  int64_t hi      = (int64_t)ceil(val);
  int64_t near    = (int64_t)nearbyint(val);
  double frac     = val - (double)lo;
  const scalar* a = &v[lo].v;
  const scalar* b = &v[hi].v;
  switch (interp) {
    case GBX_INTERP_LOWER: return value_as_double(a);
    case GBX_INTERP_HIGHER: return value_as_double(b);
    case GBX_INTERP_NEAREST: return value_as_double(&v[near].v);
    case GBX_INTERP_MIDPOINT:
      if (a->type_id == GBX_TYPE_INT64) {
        /* midpoint<double>(int64_t, int64_t), quantiles_util.hpp:65-72 */
        int64_t half = a->i / 2 + b->i / 2;
        int64_t rest = a->i % 2 + b->i % 2;
        return (double)half + (double)rest * 0.5;
      }
      return value_as_double(a) / 2 + value_as_double(b) / 2;
    default: {
      double one_minus_frac = 1.0 - frac;
      double x              = one_minus_frac * value_as_double(a);
      double y              = frac * value_as_double(b);
      return x + y;
    }
  }
}

/* MEDIAN / QUANTILE (group_quantiles.cu), NUNIQUE (group_nunique.cu) and
 * NTH_ELEMENT (group_nth_element.cu) of one request over the groups' rows,
 * rows[off[g] .. off[g+1]) in row order. */
static void finalize_sorted(gbo_column* out, const gbx_request* req, const gbx_aggregation* agg, int64_t ng,
                            const int64_t* off, const int64_t* rows)
{
  const gbx_column_view* col = &req->values;
  int32_t vt                 = value_type(col);
  int32_t tt                 = gbo_target_type(vt, agg->kind);
  int64_t nq                 = agg->kind == GBX_AGG_QUANTILE ? agg->num_quantiles : 1;
  out->type_id               = tt;
  out->scale = is_decimal(tt) ? ((col->type_id == GBX_TYPE_DICTIONARY32) ? col->dict_keys->scale : col->scale) : 0;
  out->size  = ng * nq;
  out->data  = xcalloc((size_t)(ng * nq), (size_t)type_width(tt));
  int64_t maxlen = 1;
  for (int64_t g = 0; g < ng; ++g)
    if (off[g + 1] - off[g] > maxlen) maxlen = off[g + 1] - off[g];
  sorted_value* sv = (sorted_value*)xcalloc((size_t)maxlen, sizeof(sorted_value));

  if (agg->kind == GBX_AGG_NTH_ELEMENT) {
    uint8_t* valid = (uint8_t*)xcalloc((size_t)(ng ? ng : 1), 1);
    int any_null   = 0;
    int64_t nth    = agg->ddof;
    for (int64_t g = 0; g < ng; ++g) {
      /* the group's rows, null values dropped under EXCLUDE */
      int64_t len = 0;
      for (int64_t i = off[g]; i < off[g + 1]; ++i)
        if (agg->null_policy == GBX_NULL_INCLUDE || col_valid(col, rows[i])) sv[len++].row = rows[i];
      int64_t idx = nth < 0 ? len + nth : nth;
      if (idx >= 0 && idx < len && col_valid(col, sv[idx].row)) {
        scalar v  = read_value(col, sv[idx].row);
        v.type_id = tt;
        store_scalar(out->data, tt, g, &v);
        valid[g] = 1;
      } else any_null = 1;
    }
    if (any_null) out->valid = valid;
    else free(valid);
    free(sv);
    return;
  }

  if (agg->kind == GBX_AGG_NUNIQUE) {
    for (int64_t g = 0; g < ng; ++g) {
      int64_t len = 0;
      int nulls   = 0;
      for (int64_t i = off[g]; i < off[g + 1]; ++i) {
        if (!col_valid(col, rows[i])) {
          nulls = 1;
          continue;
        }
        sv[len].v   = read_value(col, rows[i]);
        sv[len].row = rows[i];
        ++len;
      }
      qsort(sv, (size_t)len, sizeof(sorted_value), sorted_value_cmp);
      int32_t c = 0;
      for (int64_t i = 0; i < len; ++i)
        if (i == 0 || value_cmp(&sv[i].v, &sv[i - 1].v) != 0) ++c;
      if (nulls && agg->null_policy == GBX_NULL_INCLUDE) ++c;
      ((int32_t*)out->data)[g] = c;
    }
    free(sv);
    return;
  }

  /* MEDIAN = QUANTILE {0.5}, LINEAR (aggregate.cpp:344-362); always nullable */
  out->valid = (uint8_t*)xcalloc((size_t)(ng * nq > 0 ? ng * nq : 1), 1);
  for (int64_t g = 0; g < ng; ++g) {
    int64_t len = 0;
    for (int64_t i = off[g]; i < off[g + 1]; ++i) {
      if (!col_valid(col, rows[i])) continue;
      sv[len].v   = read_value(col, rows[i]);
      sv[len].row = rows[i];
      ++len;
    }
    qsort(sv, (size_t)len, sizeof(sorted_value), sorted_value_cmp);
    for (int64_t j = 0; j < nq; ++j) {
      if (len == 0) continue;
      double q       = agg->kind == GBX_AGG_MEDIAN ? 0.5 : agg->quantiles[j];
      int32_t interp = agg->kind == GBX_AGG_MEDIAN ? GBX_INTERP_LINEAR : agg->interpolation;
      ((double*)out->data)[g * nq + j] = select_quantile(sv, len, q, interp);
      out->valid[g * nq + j]            = 1;
    }
  }
  free(sv);
}

int gbo_groupby(const gbx_table_view* keys,
                int32_t null_policy,
                const gbx_request* requests,
                int32_t num_requests,
                int32_t threads,
                gbo_result** out)
{
  g_err[0] = 0;
  *out     = NULL;
  int st   = validate(keys, requests, num_requests);
  if (st != GBX_OK) return st;
  if (threads < 1) threads = 1;
  int64_t n = keys->columns[0].size;

  int keys_have_nulls = 0;
  for (int c = 0; c < keys->num_columns && !keys_have_nulls; ++c) {
    const gbx_column_view* k = &keys->columns[c];
    if (k->null_mask)
      for (int64_t r = 0; r < n && !keys_have_nulls; ++r) keys_have_nulls = !col_valid(k, r);
  }

  worker* ws   = (worker*)xcalloc((size_t)threads, sizeof(worker));
  pthread_t* tids = (pthread_t*)xcalloc((size_t)threads, sizeof(pthread_t));
  for (int t = 0; t < threads; ++t) {
    ws[t].keys           = keys;
    ws[t].null_policy    = null_policy;
    ws[t].requests       = requests;
    ws[t].num_requests   = num_requests;
    ws[t].num_rows       = n;
    ws[t].skip_null_keys = keys_have_nulls && null_policy == GBX_NULL_EXCLUDE;
    ws[t].check_nulls    = keys_have_nulls;
    ws[t].part           = t;
    ws[t].nparts         = threads;
  }
  if (threads == 1) run_worker(&ws[0]);
  else {
    for (int t = 0; t < threads; ++t) pthread_create(&tids[t], NULL, run_worker, &ws[t]);
    for (int t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
  }
  int64_t ng = 0;
  for (int t = 0; t < threads; ++t) {
    if (ws[t].status != GBX_OK) st = ws[t].status;
    ng += ws[t].num_groups;
  }

  gbo_result* r = (gbo_result*)xcalloc(1, sizeof(gbo_result));
  if (st == GBX_OK) {
    r->num_groups      = ng;
    r->num_key_columns = keys->num_columns;
    r->num_requests    = num_requests;
    int64_t* rep       = (int64_t*)xcalloc((size_t)ng, sizeof(int64_t));
    accum*** pg        = (accum***)xcalloc((size_t)(num_requests ? num_requests : 1), sizeof(accum**));
    for (int q = 0; q < num_requests; ++q) pg[q] = (accum**)xcalloc((size_t)ng, sizeof(accum*));
    int64_t g0 = 0;
    for (int t = 0; t < threads; ++t) {
      for (int64_t g = 0; g < ws[t].num_groups; ++g) {
        rep[g0 + g] = ws[t].rep_row[g];
        for (int q = 0; q < num_requests; ++q) pg[q][g0 + g] = &ws[t].acc[q][g];
      }
      g0 += ws[t].num_groups;
    }
    /* output keys: gathered from representative rows (hash/groupby.cu:607-612) */
    r->keys = (gbo_column*)xcalloc((size_t)keys->num_columns, sizeof(gbo_column));
    for (int c = 0; c < keys->num_columns; ++c) {
      const gbx_column_view* kc = &keys->columns[c];
      gbo_column* oc            = &r->keys[c];
      oc->type_id               = kc->type_id;
      oc->scale                 = kc->scale;
      oc->size                  = ng;
      if (kc->type_id == GBX_TYPE_DICTIONARY32) {
        oc->data = xcalloc((size_t)ng, 4);
        for (int64_t g = 0; g < ng; ++g) ((int32_t*)oc->data)[g] = (int32_t)dict_index(kc, rep[g]);
      } else if (kc->type_id == GBX_TYPE_STRING) {
        /* the representative rows' strings (a null key's is empty) */
        oc->str_offsets = (int64_t*)xcalloc((size_t)ng + 1, sizeof(int64_t));
        int64_t total   = 0;
        for (int64_t g = 0; g < ng; ++g) {
          int64_t len = 0;
          if (col_valid(kc, rep[g])) (void)str_at(kc, rep[g], &len);
          oc->str_offsets[g] = total;
          total += len;
        }
        oc->str_offsets[ng] = total;
        oc->data            = xcalloc((size_t)(total ? total : 1), 1);
        for (int64_t g = 0; g < ng; ++g) {
          int64_t len = 0;
          if (!col_valid(kc, rep[g])) continue;
          const unsigned char* s = str_at(kc, rep[g], &len);
          if (len) memcpy((unsigned char*)oc->data + oc->str_offsets[g], s, (size_t)len);
        }
      } else {
        oc->data = xcalloc((size_t)ng, (size_t)type_width(kc->type_id));
        for (int64_t g = 0; g < ng; ++g) {
          scalar s = read_fixed(kc, rep[g]);
          store_scalar(oc->data, kc->type_id, g, &s);
        }
      }
      if (keys_have_nulls && kc->null_mask) {
        oc->valid = (uint8_t*)xcalloc((size_t)ng, 1);
        for (int64_t g = 0; g < ng; ++g) oc->valid[g] = (uint8_t)col_valid(kc, rep[g]);
      }
    }
    /* each group's rows in row order, for the sort-path kinds */
    int64_t* goff  = NULL;
    int64_t* grows = NULL;
    int any_sorted = 0;
    for (int q = 0; q < num_requests; ++q)
      for (int k = 0; k < requests[q].num_aggregations; ++k)
        any_sorted |= is_sorted_kind(requests[q].aggregations[k].kind);
    if (any_sorted) {
      int64_t* base = (int64_t*)xcalloc((size_t)threads, sizeof(int64_t));
      for (int t = 1; t < threads; ++t) base[t] = base[t - 1] + ws[t - 1].num_groups;
      int64_t* gid = (int64_t*)xcalloc((size_t)(n ? n : 1), sizeof(int64_t));
      goff         = (int64_t*)xcalloc((size_t)(ng + 1), sizeof(int64_t));
      for (int64_t row = 0; row < n; ++row) {
        gid[row] = -1;
        for (int t = 0; t < threads; ++t)
          if (ws[t].row_gid[row] >= 0) gid[row] = base[t] + ws[t].row_gid[row];
        if (gid[row] >= 0) goff[gid[row] + 1]++;
      }
      for (int64_t g = 0; g < ng; ++g) goff[g + 1] += goff[g];
      grows        = (int64_t*)xcalloc((size_t)(goff[ng] ? goff[ng] : 1), sizeof(int64_t));
      int64_t* pos = (int64_t*)xcalloc((size_t)(ng ? ng : 1), sizeof(int64_t));
      for (int64_t row = 0; row < n; ++row)
        if (gid[row] >= 0) grows[goff[gid[row]] + pos[gid[row]]++] = row;
      free(pos);
      free(gid);
      free(base);
    }
    r->num_results = (int32_t*)xcalloc((size_t)(num_requests ? num_requests : 1), sizeof(int32_t));
    r->results = (gbo_column**)xcalloc((size_t)(num_requests ? num_requests : 1), sizeof(gbo_column*));
    for (int q = 0; q < num_requests; ++q) {
      const gbx_request* rq = &requests[q];
      r->num_results[q]     = rq->num_aggregations;
      r->results[q] = (gbo_column*)xcalloc((size_t)(rq->num_aggregations ? rq->num_aggregations : 1),
                                           sizeof(gbo_column));
      for (int k = 0; k < rq->num_aggregations; ++k) {
        if (is_sorted_kind(rq->aggregations[k].kind))
          finalize_sorted(&r->results[q][k], rq, &rq->aggregations[k], ng, goff, grows);
        else finalize_column(&r->results[q][k], rq, &rq->aggregations[k], ng, pg[q], rep);
      }
    }
    free(goff);
    free(grows);
    for (int q = 0; q < num_requests; ++q) free(pg[q]);
    free(pg);
    free(rep);
  } else {
    free(r);
    r = NULL;
    set_err(st, "oracle worker failed (%d)", st);
  }
  for (int t = 0; t < threads; ++t) {
    free(ws[t].rep_row);
    free(ws[t].row_gid);
    if (ws[t].acc) {
      for (int q = 0; q < num_requests; ++q) free(ws[t].acc[q]);
      free(ws[t].acc);
    }
  }
  free(ws);
  free(tids);
  *out = r;
  return st;
}

void gbo_result_free(gbo_result* r)
{
  if (!r) return;
  for (int c = 0; c < r->num_key_columns; ++c) {
    free(r->keys[c].data);
    free(r->keys[c].valid);
    free(r->keys[c].str_offsets);
  }
  free(r->keys);
  for (int q = 0; q < r->num_requests; ++q) {
    for (int k = 0; k < r->num_results[q]; ++k) {
      free(r->results[q][k].data);
      free(r->results[q][k].valid);
    }
    free(r->results[q]);
  }
  free(r->results);
  free(r->num_results);
  free(r);
}
