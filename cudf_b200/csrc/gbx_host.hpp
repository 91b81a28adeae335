// gbx_host.hpp -- host-side building blocks shared by libgbx's entry points
// (the plain groupby in gbx_abi.cpp, the batched form in gbx_batch.cpp, the
// served form in gbx_server.cpp): error reporting, type rules, allocation,
// and lowering of a groupby call to a Plan (packed keys, value channels and
// their accumulators).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <new>
#include <string>
#include <utility>
#include <deque>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_kernels.hpp"

namespace gbx {

// ------------------------------------------------------------------ errors

extern thread_local std::string g_last_error;

struct Failure {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const char* fmt, ...);

#define GBX_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      if (e_ == cudaErrorMemoryAllocation)                                                  \
        ::gbx::fail(GBX_ERR_ALLOC, "CUDA error at %s:%d: %s", __FILE__, __LINE__,           \
                    cudaGetErrorString(e_));                                                \
      ::gbx::fail(GBX_ERR_CUDA, "CUDA error at %s:%d: %s", __FILE__, __LINE__,              \
                  cudaGetErrorString(e_));                                                  \
    }                                                                                       \
  } while (0)

#define GBX_EXPECTS(cond, ...)                            \
  do {                                                    \
    if (!(cond)) ::gbx::fail(GBX_ERR_LOGIC, __VA_ARGS__); \
  } while (0)

// Runs `f`, turning a Failure into a status code and the thread's message.
// A non-sticky error left in the thread's CUDA error state by an earlier,
// unrelated call is cleared first, so that the launch checks inside `f`
// (cudaGetLastError) only see this call's own launches.
template <class F>
int guarded(F&& f)
{
  (void)cudaGetLastError();
  try {
    f();
    g_last_error.clear();
    return GBX_OK;
  } catch (Failure& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return GBX_ERR_ALLOC;
  }
}

// -------------------------------------------------------------- type rules

int type_width(int32_t t);
bool is_integral(int32_t t);
bool is_floating(int32_t t);
bool is_duration(int32_t t);
bool is_decimal(int32_t t);
bool is_fixed_width(int32_t t);
bool is_unsigned(int32_t t);
int8_t phys_of(int32_t t);
int32_t target_type(int32_t t, int32_t kind);
bool is_hash_kind(int32_t k);
// MEDIAN / QUANTILE / NUNIQUE / NTH_ELEMENT (computed by gbx_sort.cu)
bool is_sort_kind(int32_t k);
// the kinds the batched form computes
bool is_batch_kind(int32_t k);
int32_t value_type(const gbx_column_view& c);
bool same_view(const gbx_column_view& a, const gbx_column_view& b);

// -------------------------------------------------------------- allocation

// Device allocations through the caller's allocator, else stream-ordered
// cudaMallocAsync.
struct Alloc {
  gbx_allocator user{};
  bool has_user   = false;
  cudaStream_t st = nullptr;

  void* allocate(size_t bytes);
  void release(void* p, size_t bytes);
};

// Scratch buffers released (stream-ordered) when the owner goes away.
struct Scratch {
  Alloc* a;
  std::vector<std::pair<void*, size_t>> bufs;
  explicit Scratch(Alloc* al) : a(al) {}
  Scratch(const Scratch&)            = delete;
  Scratch& operator=(const Scratch&) = delete;
  void* get(size_t bytes)
  {
    void* p = a->allocate(bytes);
    bufs.emplace_back(p, bytes);
    return p;
  }
  size_t total() const
  {
    size_t s = 0;
    for (auto& b : bufs) s += b.second;
    return s;
  }
  void release_all()
  {
    for (auto& b : bufs) a->release(b.first, b.second);
    bufs.clear();
  }
  ~Scratch() { release_all(); }
};

struct DeviceInfo {
  int device        = -1;
  int num_sms       = 0;
  size_t smem_optin = 0;
  size_t l2_bytes   = 0;
};

DeviceInfo current_device();
uint64_t next_pow2(uint64_t v);

// Allocates an output column of `n` rows (plus a padded bitmask).
void alloc_column(Alloc& a, gbx_column& c, int32_t type_id, int32_t scale, int64_t n, bool with_mask);

}  // namespace gbx

// gbx_result::internal: the allocator the result's buffers go back to
// (gbx_result_release).
// Releases a result when it goes out of scope unless taken: the error paths
// of the calls that build one result from another.
struct ResultHold {
  gbx_result* r = nullptr;
  ResultHold() = default;
  ResultHold(const ResultHold&) = delete;
  ResultHold& operator=(const ResultHold&) = delete;
  ~ResultHold() { if (r) gbx_result_release(r); }
  gbx_result* take()
  {
    gbx_result* t = r;
    r             = nullptr;
    return t;
  }
};

struct ResultInternal {
  gbx::Alloc alloc;
  // buffers beyond the columns' own (STRING keys' offsets, STRUCT keys'
  // members) and the child views the columns point at
  std::vector<std::pair<void*, size_t>> extra;
  std::deque<gbx_column_view> children;
  std::deque<std::vector<gbx_column_view>> arrays;  // STRUCT members
};

namespace gbx {

// ------------------------------------------------------------------ plans

// verify_valid_requests (groupby.cu:176-192) and the size check of
// groupby::aggregate (groupby.cu:210-214) for keys of `n` rows.
// count_any: COUNT_VALID / COUNT_ALL are accepted over any value type (the
// plain entry point answers them through stand-in columns).
void validate_requests(const gbx_request* reqs, int32_t nreq, int64_t n, bool count_any = false);
bool counted_only(int32_t value_type);

// Keys that do not pack into two 64-bit words (STRING columns, or more than
// 128 bits with the null bits) and the groupby over them: rows labelled by a
// representative-row table, the groupby run on the label (gbx_rep.cu).
bool keys_need_representatives(const std::vector<gbx_column_view>& keys, int32_t null_policy);
int aggregate_by_representatives(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                                 const gbx_request* requests, int32_t num_requests, void* stream,
                                 const gbx_allocator* mr, gbx_result** out, gbx_stats* stats);
// Distinct rows of STRING / STRUCT keys through representative rows
// (gbx_join.cu): the kept row indices into *out (when not null); returns
// their number.
bool keys_are_nested_or_strings(const gbx_table_view* keys);
int64_t distinct_by_representatives(const gbx_table_view* keys, int32_t keep, int32_t nulls_equal,
                                    int32_t nans_equal, void* stream, const gbx_allocator* mr, gbx_column* out);
// MIN / MAX of STRING values (gbx_rep.cu): each group's least / greatest
// string by a compare-and-swap of its best row, the other requests by the
// groupby on the key's representative-row label.
bool needs_string_extrema(const gbx_request* requests, int32_t num_requests);
int aggregate_string_extrema(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                             const gbx_request* requests, int32_t num_requests, void* stream,
                             const gbx_allocator* mr, gbx_result** out, gbx_stats* stats);
// The strategy set on a groupby (a groupby run on labels inherits it).
int32_t groupby_strategy(const gbx_groupby* gb);
// Keys the caller declares sorted: groups are the runs of equal adjacent rows
// in row order; under EXCLUDE with null keys, one group per key ordered by
// its first row (gbx_rep.cu).
int aggregate_presorted(gbx_groupby* gb, const std::vector<gbx_column_view>& keys, int32_t null_policy,
                        const gbx_request* requests, int32_t num_requests, void* stream, const gbx_allocator* mr,
                        gbx_result** out, gbx_stats* stats);

// ARGMIN / ARGMAX over values of up to 32 bits as MIN / MAX of packed words
// (gbx_args.cu): whether the requests hold such kinds only, and the groupby
// with them rewritten.
bool args_packable(const gbx_request* requests, int32_t num_requests);
// Requests whose values only COUNT can read (STRING, LIST, STRUCT,
// DECIMAL128): answered over an INT8 stand-in with the same rows and
// validity (gbx_args.cu).
bool needs_count_stand_ins(const gbx_request* requests, int32_t num_requests);
int aggregate_with_count_stand_ins(gbx_groupby* gb, int64_t n, const gbx_request* requests, int32_t num_requests,
                                   void* stream, const gbx_allocator* mr, gbx_result** out);
int aggregate_with_packed_args(gbx_groupby* gb, int64_t n, const gbx_request* requests, int32_t num_requests,
                               void* stream, const gbx_allocator* mr, gbx_result** out);
int8_t phys_of(int32_t t);

// Null count of a column when known without a kernel (0 without a mask), else -1.
int64_t exact_null_count_or_neg(const gbx_column_view& c);

// Byte layout of one shared-memory table of S + 1 slots.
SmemLayout make_smem_layout(const Plan& plan, uint32_t S);

// Packs the key columns into one or two 64-bit words.  `key_nulls[c]` is the
// null count of key column c (or -1: unknown, treated as nullable).  `ok` is
// false when the keys need more than 128 bits.
KeyPlan make_key_plan(const gbx_column_view* keys, int nkeys, int32_t null_policy,
                      const std::vector<int64_t>& key_nulls, bool& ok);

// The distinct value columns of the requests (one channel each); req_chan[q]
// is request q's channel (-1 for a request without aggregations).
std::vector<const gbx_column_view*> collect_channels(const gbx_request* reqs, int32_t nreq,
                                                     std::vector<int>& req_chan);

// Fills plan.nchan, plan.chan and plan.acc for the channels and the
// aggregations that use them (flatten_single_pass_aggs, hash/groupby.cu:351-383).
// A channel gets its own valid count when chan_nulls[c] != 0.
void fill_channels(Plan& plan, const std::vector<const gbx_column_view*>& chan_cols,
                   const std::vector<int64_t>& chan_nulls, const gbx_request* reqs, int32_t nreq,
                   const std::vector<int>& req_chan);

// Group count of `n` rows from a sample of `sampled` rows with `distinct`
// distinct keys (uniform-draw inversion, clamped to [1, n]).
double estimate_groups(double sampled, double distinct, int64_t n, int64_t nsample);
// The same with the sample's `heavy` frequent keys (and their `heavy_rows`
// sampled rows) counted exactly and the inversion applied to the remaining
// rows only, so that a few frequent keys do not hide many rare ones.
double estimate_groups(double sampled, double distinct, double heavy, double heavy_rows, int64_t n, int64_t nsample);

// Bytes of one table slot: packed key, row count and every accumulator.
size_t slot_bytes(const Plan& plan);

}  // namespace gbx
