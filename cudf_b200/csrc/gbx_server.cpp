// gbx_server.cpp -- the served groupby (include/gbx.h, gbx_server_*):
// continuous batching of groupby requests over device-resident columns.
//
// Requests wait in arrival order.  A worker (one host thread and one CUDA
// stream each) that becomes free admits the first waiting request whose
// memory charge fits the HBM budget beside the admitted ones; when that
// request is small, the other waiting small requests of the same schema that
// fit go with it into one batched launch (gbx_batch, one shot).  Workers run
// concurrently, so requests that arrive while others are on the GPU start as
// soon as a worker and memory are free, and their kernels overlap on the
// device.  A single request runs through gbx_groupby_aggregate -- the
// reference's groupby::aggregate path (groupby.cu:197-221) -- so its result
// is the plain form's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_host.hpp"
#include "gbx_kernels.hpp"

using namespace gbx;

namespace gbx {
namespace {

// A request with its own copies of every descriptor it was submitted with.
struct Job {
  uint64_t ticket = 0;
  std::vector<gbx_column_view> keys;
  std::vector<gbx_column_view> key_dicts;
  std::vector<gbx_request> reqs;
  std::vector<std::vector<gbx_aggregation>> aggs;
  std::vector<std::vector<double>> quantiles;  // copies of QUANTILE arrays (aggs point here)
  std::vector<gbx_column_view> val_dicts;
  int64_t rows   = 0;
  int64_t charge = 0;
  std::string schema;  // requests with equal strings may share a batched launch
  double submitted = 0, admitted = 0, done = 0;
  int status = GBX_OK;
  std::string error;
  gbx_result* result = nullptr;
  int batched        = 1;
  int worker         = -1;
  bool finished      = false;
  bool mergeable     = true;  // dictionary keys never share a batched launch
  bool large         = false;  // at least opt.large_rows rows
};

// Device bytes a request may hold at once on the plain path, bounded from
// above: packed keys and value copies of the partitioned path, tables sized
// for every row being its own group (the overflow retry's size) with their
// compaction map, and outputs for that many groups.
int64_t memory_charge(const Job& j)
{
  int64_t key_bytes = 0, null_bits = 0;
  for (auto& k : j.keys) {
    key_bytes += type_width(k.type_id == GBX_TYPE_DICTIONARY32 ? GBX_TYPE_INT32 : k.type_id);
    null_bits += k.null_mask ? 1 : 0;
  }
  const int64_t nw = (key_bytes * 8 + null_bits > 64) ? 16 : 8;  // packed key words
  int64_t val_copy = 0, acc = 4, out = key_bytes + 1, sorted = 0;
  for (size_t q = 0; q < j.reqs.size(); ++q) {
    const int32_t vt = value_type(j.reqs[q].values);
    val_copy += type_width(vt) + 1;
    for (auto& a : j.aggs[q]) {
      acc += 16;  // at most two 8-byte accumulators per aggregation
      const int64_t per_group = a.kind == GBX_AGG_QUANTILE ? std::max(a.num_quantiles, 1) : 1;
      out += per_group * (std::max(4, type_width(target_type(vt, a.kind))) + 1);
      // the sorted kinds: row labels, two record buffers and the flags
      if (is_sort_kind(a.kind)) sorted = 44;
    }
  }
  const int64_t n = std::max<int64_t>(j.rows, 1);
  return n * (nw + val_copy + sorted) + 4 * n * (nw + acc + 4) + n * out + (int64_t(32) << 20);
}

std::string schema_of(const Job& j)
{
  std::ostringstream os;
  for (auto& k : j.keys) os << 'k' << k.type_id << ':' << k.scale;
  for (size_t q = 0; q < j.reqs.size(); ++q) {
    const gbx_column_view& v = j.reqs[q].values;
    os << "|v" << v.type_id << ':' << v.scale << ':' << v.index_type_id;
    if (v.type_id == GBX_TYPE_DICTIONARY32 && v.dict_keys) os << 'd' << v.dict_keys->type_id;
    for (auto& a : j.aggs[q]) os << ',' << a.kind << '/' << a.ddof;
  }
  return os.str();
}

}  // namespace
}  // namespace gbx

struct gbx_server {
  gbx_server_options opt{};
  int device = 0;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work;
  std::condition_variable cv_done;
  std::deque<std::shared_ptr<Job>> waiting;
  std::unordered_map<uint64_t, std::shared_ptr<Job>> jobs;
  uint64_t next_ticket = 1;
  int64_t reserved     = 0;
  int in_flight        = 0;
  int large_in_flight  = 0;
  bool stopping        = false;
  double busy_since    = 0;
  gbx_server_stats st{};
  std::vector<std::thread> threads;

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace gbx {
namespace {

// Picks the next launch under the lock: the first waiting request whose
// charge fits and, when it is large, while fewer than opt.large_in_flight
// large requests run (a large request fills the GPU by itself: two of them
// only interleave their kernels and evict each other's L2-resident tables);
// small ones take the waiting small requests of their schema along.  Empty
// when nothing fits.
std::vector<std::shared_ptr<Job>> pick(gbx_server& s)
{
  std::vector<std::shared_ptr<Job>> out;
  const int64_t budget = s.opt.hbm_budget_bytes;
  for (auto it = s.waiting.begin(); it != s.waiting.end(); ++it) {
    const auto j = *it;
    if (j->large && s.large_in_flight >= s.opt.large_in_flight) continue;
    const bool alone_ok = s.in_flight == 0 && s.reserved == 0;  // larger than the budget: runs alone
    if (s.reserved + j->charge > budget && !(j->charge > budget && alone_ok)) continue;
    out.push_back(j);
    int64_t charged = j->charge;
    s.waiting.erase(it);
    if (s.opt.batch_max_rows > 0 && j->mergeable && j->rows <= s.opt.batch_max_rows) {
      for (auto jt = s.waiting.begin(); jt != s.waiting.end() && static_cast<int>(out.size()) < s.opt.batch_max_requests;) {
        const auto& k = *jt;
        if (k->mergeable && k->rows <= s.opt.batch_max_rows && k->schema == j->schema &&
            s.reserved + charged + k->charge <= budget) {
          charged += k->charge;
          out.push_back(k);
          jt = s.waiting.erase(jt);
        } else {
          ++jt;
        }
      }
    }
    break;
  }
  return out;
}

gbx_table_view table_of(Job& j)
{
  gbx_table_view tv{};
  tv.num_columns = static_cast<int32_t>(j.keys.size());
  tv.columns     = j.keys.data();
  return tv;
}

// One request alone: the plain form on this worker's stream.
void run_single(gbx_server& s, Job& j, cudaStream_t st)
{
  gbx_table_view tv = table_of(j);
  gbx_groupby* gb   = nullptr;
  int rc            = gbx_groupby_create(&tv, s.opt.null_policy, 0, &gb);
  gbx_result* res   = nullptr;
  if (rc == GBX_OK) rc = gbx_groupby_aggregate(gb, j.reqs.data(), static_cast<int32_t>(j.reqs.size()), st, nullptr, &res);
  if (rc != GBX_OK) j.error = gbx_last_error();
  if (gb) gbx_groupby_destroy(gb);
  // the call synchronised its stream: the caller may free on any stream
  if (res) static_cast<ResultInternal*>(res->internal)->alloc.st = nullptr;
  j.status = rc;
  j.result = res;
}

// Copies rows [off, off + n) of a batch output column into a new column.
void slice_column(Alloc& a, const gbx_column& src, int64_t off, int64_t n, gbx_column& dst, cudaStream_t st)
{
  const gbx_column_view& v = src.view;
  alloc_column(a, dst, v.type_id, v.scale, n, src.null_mask != nullptr);
  const int w = type_width(v.type_id);
  if (n > 0) {
    GBX_CUDA(cudaMemcpyAsync(dst.data, static_cast<const char*>(src.data) + off * w, static_cast<size_t>(n) * w,
                             cudaMemcpyDeviceToDevice, st));
    if (src.null_mask) GBX_CUDA(launch_copy_bits(src.null_mask, off, dst.null_mask, n, st));
  }
  dst.view.null_count = 0;
}

// Several small requests of one schema: one one-shot batched launch, then
// each request's rows copied out into its own result.
void run_merged(gbx_server& s, std::vector<std::shared_ptr<Job>>& js, cudaStream_t st, int num_sms)
{
  const int m = static_cast<int>(js.size());
  std::vector<gbx_batch_instance> inst(m);
  for (int i = 0; i < m; ++i) {
    inst[i].keys     = table_of(*js[i]);
    inst[i].requests = js[i]->reqs.data();
  }
  gbx_batch_options o{};
  o.null_policy  = s.opt.null_policy;
  o.tune         = GBX_TUNE_OFF;
  o.one_shot     = 1;
  gbx_batch* b   = nullptr;
  const int nreq = static_cast<int>(js[0]->reqs.size());
  int rc         = gbx_batch_create(inst.data(), m, nreq, &o, st, nullptr, &b);
  const gbx_batch_output* out = nullptr;
  if (rc == GBX_OK) rc = gbx_batch_execute(b, st, &out);
  if (rc != GBX_OK) {
    // one launch per request instead (each then reports its own error)
    if (b) gbx_batch_destroy(b);
    for (auto& j : js) run_single(s, *j, st);
    return;
  }
  unsigned long long* d_valid = nullptr;
  Alloc a;
  a.st    = st;
  int err = guarded([&] {
    const gbx_result& cols = out->columns;
    std::vector<unsigned long long> h_valid(kMaxMaskSpans, 0);
    d_valid = static_cast<unsigned long long*>(a.allocate(kMaxMaskSpans * 8));
    for (int i = 0; i < m; ++i) {
      const int64_t off = out->group_offsets[i], n = out->group_offsets[i + 1] - off;
      auto* res = new gbx_result();
      std::memset(res, 0, sizeof(*res));
      res->internal        = new ResultInternal{Alloc{}};
      res->num_groups      = n;
      res->num_key_columns = cols.num_key_columns;
      res->num_requests    = cols.num_requests;
      res->keys            = new gbx_column[std::max(1, cols.num_key_columns)]();
      res->requests        = new gbx_aggregation_result[std::max(1, cols.num_requests)]();
      js[i]->result        = res;
      MaskSpans ms{};
      std::vector<gbx_column*> masked;
      for (int c = 0; c < cols.num_key_columns; ++c) {
        slice_column(a, cols.keys[c], off, n, res->keys[c], st);
        if (res->keys[c].null_mask) {
          ms.span[ms.n++] = MaskSpan{res->keys[c].null_mask, 0, n};
          masked.push_back(&res->keys[c]);
        }
      }
      for (int q = 0; q < cols.num_requests; ++q) {
        const gbx_aggregation_result& ar = cols.requests[q];
        res->requests[q].num_results     = ar.num_results;
        res->requests[q].results         = new gbx_column[std::max(1, ar.num_results)]();
        for (int k = 0; k < ar.num_results; ++k) {
          slice_column(a, ar.results[k], off, n, res->requests[q].results[k], st);
          if (res->requests[q].results[k].null_mask) {
            if (ms.n == kMaxMaskSpans) fail(GBX_ERR_UNSUPPORTED, "too many nullable outputs to merge");
            ms.span[ms.n++] = MaskSpan{res->requests[q].results[k].null_mask, 0, n};
            masked.push_back(&res->requests[q].results[k]);
          }
        }
      }
      if (ms.n > 0 && n > 0) {
        GBX_CUDA(cudaMemsetAsync(d_valid, 0, kMaxMaskSpans * 8, st));
        GBX_CUDA(launch_count_valid(ms, d_valid, num_sms, st));
        GBX_CUDA(cudaMemcpyAsync(h_valid.data(), d_valid, kMaxMaskSpans * 8, cudaMemcpyDeviceToHost, st));
        GBX_CUDA(cudaStreamSynchronize(st));
        for (int c = 0; c < ms.n; ++c) masked[c]->view.null_count = n - static_cast<int64_t>(h_valid[c]);
      }
    }
    GBX_CUDA(cudaStreamSynchronize(st));
  });
  if (d_valid) a.release(d_valid, kMaxMaskSpans * 8);
  const std::string msg = err == GBX_OK ? std::string() : gbx_last_error();
  gbx_batch_destroy(b);
  for (auto& j : js) {
    j->status  = err;
    j->error   = msg;
    j->batched = m;
    if (err != GBX_OK && j->result) {
      gbx_result_release(j->result);
      j->result = nullptr;
    }
  }
}

void worker_main(gbx_server* s, int w)
{
  cudaSetDevice(s->device);
  // small requests on a high-priority stream, large ones on a low-priority
  // one: blocks of a small request's kernels are scheduled ahead of a large
  // request's waiting blocks
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  cudaStream_t st = nullptr, st_large = nullptr;
  cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_hi);
  cudaStreamCreateWithPriority(&st_large, cudaStreamNonBlocking, prio_lo);
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    std::vector<std::shared_ptr<Job>> js;
    s->cv_work.wait(lk, [&] {
      if (s->stopping) return true;
      js = pick(*s);
      return !js.empty();
    });
    if (js.empty()) break;  // stopping
    const double t = s->now();
    int64_t charge = 0;
    for (auto& j : js) {
      j->admitted = t;
      j->worker   = w;
      charge += j->charge;
    }
    s->reserved += charge;
    if (s->in_flight++ == 0) s->busy_since = t;
    const bool large = js.size() == 1 && js[0]->large;
    if (large) s->large_in_flight += 1;
    s->st.max_in_flight       = std::max(s->st.max_in_flight, s->in_flight);
    s->st.peak_reserved_bytes = std::max(s->st.peak_reserved_bytes, s->reserved);
    lk.unlock();

    if (js.size() == 1) run_single(*s, *js[0], large ? st_large : st);
    else run_merged(*s, js, st, num_sms);

    lk.lock();
    const double d = s->now();
    s->reserved -= charge;
    if (large) s->large_in_flight -= 1;
    if (--s->in_flight == 0) s->st.busy_s += d - s->busy_since;
    if (js.size() > 1) {
      s->st.batches += 1;
      s->st.batched_requests += static_cast<int64_t>(js.size());
    }
    for (auto& j : js) {
      j->done     = d;
      j->finished = true;
      if (j->status == GBX_OK) {
        s->st.completed += 1;
        s->st.rows += j->rows;
      } else {
        s->st.failed += 1;
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();  // memory came back: others may fit now
  }
  lk.unlock();
  cudaStreamSynchronize(st);
  cudaStreamSynchronize(st_large);
  cudaStreamDestroy(st);
  cudaStreamDestroy(st_large);
}

}  // namespace
}  // namespace gbx

extern "C" {

int gbx_server_create(const gbx_server_options* options, gbx_server** out)
{
  gbx_server* s = nullptr;
  int rc        = guarded([&] {
    GBX_EXPECTS(out != nullptr, "out is null");
    *out = nullptr;
    gbx_server_options o{};
    if (options) o = *options;
    if (o.workers == 0) o.workers = 4;
    if (o.hbm_budget_bytes == 0) o.hbm_budget_bytes = int64_t(150) << 30;
    if (o.batch_max_requests == 0) o.batch_max_requests = 64;
    if (o.large_in_flight == 0) o.large_in_flight = 1;
    if (o.large_rows == 0) o.large_rows = int64_t(1) << 22;
    GBX_EXPECTS(o.workers >= 1 && o.workers <= 256, "workers must be in [1, 256]");
    GBX_EXPECTS(o.large_in_flight >= 1, "large_in_flight must be >= 1");
    GBX_EXPECTS(o.null_policy == GBX_NULL_EXCLUDE || o.null_policy == GBX_NULL_INCLUDE, "invalid null_policy");
    GBX_EXPECTS(o.hbm_budget_bytes > 0 && o.batch_max_rows >= 0 && o.batch_max_requests >= 1,
                "invalid budget or batching limits");
    s      = new gbx_server();
    s->opt = o;
    s->t0  = std::chrono::steady_clock::now();
    GBX_CUDA(cudaGetDevice(&s->device));
    // requests allocate from this process's default stream-ordered pool; let
    // it keep up to the budget cached between requests instead of returning
    // memory to the driver at every synchronisation
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
      uint64_t keep = static_cast<uint64_t>(o.hbm_budget_bytes);
      GBX_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    s->st.workers = o.workers;
    for (int w = 0; w < o.workers; ++w) s->threads.emplace_back(worker_main, s, w);
    *out = s;
  });
  if (rc != GBX_OK && s) gbx_server_destroy(s);
  return rc;
}

int gbx_server_submit(gbx_server* s, const gbx_table_view* keys, const gbx_request* requests, int32_t num_requests,
                      uint64_t* ticket)
{
  return guarded([&] {
    GBX_EXPECTS(s != nullptr && keys != nullptr && ticket != nullptr, "null argument");
    GBX_EXPECTS(keys->num_columns >= 1 && keys->columns != nullptr, "a request needs key columns");
    auto j = std::make_shared<Job>();
    j->keys.assign(keys->columns, keys->columns + keys->num_columns);
    j->key_dicts.resize(j->keys.size());
    for (size_t c = 0; c < j->keys.size(); ++c) {
      if (j->keys[c].type_id == GBX_TYPE_STRUCT)
        fail(GBX_ERR_UNSUPPORTED, "STRUCT keys are not served; use gbx_groupby_aggregate");
      if (j->keys[c].dict_keys) {
        j->key_dicts[c]      = *j->keys[c].dict_keys;
        j->keys[c].dict_keys = &j->key_dicts[c];
      }
      if (j->keys[c].type_id == GBX_TYPE_DICTIONARY32 || j->keys[c].type_id == GBX_TYPE_STRING) j->mergeable = false;
      GBX_EXPECTS(j->keys[c].size == j->keys[0].size, "key columns differ in size");
    }
    j->rows = j->keys[0].size;
    validate_requests(requests, num_requests, j->rows);
    j->reqs.assign(requests, requests + num_requests);
    j->aggs.resize(num_requests);
    j->val_dicts.resize(num_requests);
    size_t nquant = 0;
    for (int q = 0; q < num_requests; ++q)
      for (int k = 0; k < requests[q].num_aggregations; ++k)
        nquant += requests[q].aggregations[k].kind == GBX_AGG_QUANTILE ? 1 : 0;
    j->quantiles.reserve(nquant);  // no reallocation: aggs keep pointers into it
    for (int q = 0; q < num_requests; ++q) {
      // ARGMIN / ARGMAX, M2 and the sorted kinds run on the plain path only
      // (the batched form lacks them)
      for (int k = 0; k < requests[q].num_aggregations; ++k)
        if (!is_batch_kind(requests[q].aggregations[k].kind)) j->mergeable = false;
      j->aggs[q].assign(requests[q].aggregations, requests[q].aggregations + requests[q].num_aggregations);
      for (gbx_aggregation& a : j->aggs[q])
        if (a.kind == GBX_AGG_QUANTILE) {
          j->quantiles.emplace_back(a.quantiles, a.quantiles + a.num_quantiles);
          a.quantiles = j->quantiles.back().data();
        }
      j->reqs[q].aggregations = j->aggs[q].data();
      if (j->reqs[q].values.dict_keys) {
        j->val_dicts[q]             = *j->reqs[q].values.dict_keys;
        j->reqs[q].values.dict_keys = &j->val_dicts[q];
      }
    }
    j->charge = memory_charge(*j);
    j->schema = schema_of(*j);
    j->large  = s->opt.large_rows > 0 && j->rows >= s->opt.large_rows;
    std::lock_guard<std::mutex> lk(s->mu);
    GBX_EXPECTS(!s->stopping, "the server is shutting down");
    j->ticket          = s->next_ticket++;
    j->submitted       = s->now();
    s->jobs[j->ticket] = j;
    s->waiting.push_back(j);
    s->st.submitted += 1;
    *ticket = j->ticket;
    s->cv_work.notify_one();
  });
}

int gbx_server_wait(gbx_server* s, uint64_t ticket, double timeout_s, gbx_result** out, gbx_server_timing* timing)
{
  std::shared_ptr<Job> j;
  int rc = guarded([&] {
    GBX_EXPECTS(s != nullptr && out != nullptr, "null argument");
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    GBX_EXPECTS(it != s->jobs.end(), "unknown ticket %llu", static_cast<unsigned long long>(ticket));
    j          = it->second;
    auto ready = [&] { return j->finished; };
    if (timeout_s < 0) {
      s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
      j.reset();
      fail(GBX_ERR_LOGIC, "timeout waiting for ticket %llu", static_cast<unsigned long long>(ticket));
    }
    s->jobs.erase(ticket);
  });
  if (rc != GBX_OK) return rc;
  if (timing) {
    timing->submitted_s    = j->submitted;
    timing->admitted_s     = j->admitted;
    timing->done_s         = j->done;
    timing->reserved_bytes = j->charge;
    timing->batched        = j->batched;
    timing->worker         = j->worker;
  }
  if (j->status != GBX_OK) {
    g_last_error = j->error;
    return j->status;
  }
  *out = j->result;
  return GBX_OK;
}

double gbx_server_now(const gbx_server* s) { return s ? s->now() : 0.0; }

int gbx_server_last_stats(const gbx_server* s, gbx_server_stats* out)
{
  return guarded([&] {
    GBX_EXPECTS(s != nullptr && out != nullptr, "null argument");
    std::lock_guard<std::mutex> lk(const_cast<gbx_server*>(s)->mu);
    *out = s->st;
  });
}

void gbx_server_destroy(gbx_server* s)
{
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (auto& j : s->waiting) {
      j->status   = GBX_ERR_LOGIC;
      j->error    = "the server was destroyed before the request ran";
      j->finished = true;
    }
    s->waiting.clear();
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  for (auto& t : s->threads) t.join();
  for (auto& kv : s->jobs)
    if (kv.second->result) gbx_result_release(kv.second->result);
  delete s;
}

}  // extern "C"
