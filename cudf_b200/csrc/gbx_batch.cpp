// gbx_batch.cpp -- host side of the batched groupby (include/gbx.h,
// gbx_batch_*): schema checks, per-instance sampling, the autotuner and its
// persisted table, the table arena and concatenated outputs, and the CUDA
// graph that runs a whole batch in one launch.
//
// Each instance computes exactly what gbx_groupby_aggregate computes on it
// alone (the reference's groupby::aggregate, groupby.cu:197-221, restated by
// gbx_abi.cpp); only the scheduling differs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/gbx.h"
#include "gbx_batch.hpp"
#include "gbx_host.hpp"

using namespace gbx;

namespace gbx {
namespace {

// Dynamic shared memory per CTA for the two block shapes the tuner picks
// from: 256 threads with two CTAs per SM, or 512 threads with one.
constexpr size_t kSmemBudget256  = 100 * 1024;
constexpr size_t kSmemBudget512  = kBatchMaxDynamicSmem;
constexpr int kSamplePerInstance = 2048;
constexpr int kMinTileLog2       = 12;
constexpr int kMaxTileLog2       = 20;

size_t smem_budget(int block) { return block == 512 ? kSmemBudget512 : kSmemBudget256; }

// One tuned choice for a class of instances under one block shape.
struct Choice {
  int32_t mode      = BM_GLOBAL;
  int32_t smul      = 0;   // shared table slots = base_slots(class) << smul
  int32_t tile_log2 = 16;  // rows per work item
  double rate       = 0;   // measured rows/s of the class (0: not measured)
};

// Tuning class of an instance: the octave of its estimated group count.
int class_of(double est)
{
  int c = 0;
  while (c < 40 && std::ldexp(1.0, c + 1) <= est) ++c;
  return c;
}

// Slots of a shared-memory table for a class at load <= 0.8 of its largest
// member (groups < 2^(cls+1)).
uint32_t base_slots(int cls)
{
  uint64_t s = next_pow2(static_cast<uint64_t>(std::ceil(std::ldexp(1.0, cls + 1) * 1.25)));
  return static_cast<uint32_t>(std::max<uint64_t>(s, 32));
}

// ---------------------------------------------------------- tuning table

std::mutex g_tune_mutex;

struct TuneKey {
  std::string device, sig;
  int block, cls;
  bool operator<(const TuneKey& o) const
  {
    return std::tie(device, sig, block, cls) < std::tie(o.device, o.sig, o.block, o.cls);
  }
};

// Lines: "<device> <schema> <block> <class> <mode> <smul> <tile_log2> <rows/s>";
// later lines override earlier ones.
std::map<TuneKey, Choice> read_tune_file(const char* path)
{
  std::map<TuneKey, Choice> m;
  if (!path || !*path) return m;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    TuneKey k;
    Choice c;
    if (!(is >> k.device >> k.sig >> k.block >> k.cls >> c.mode >> c.smul >> c.tile_log2 >> c.rate)) continue;
    if (c.mode < BM_SHARED || c.mode > BM_GLOBAL || c.smul < 0 || c.smul > 2 || c.tile_log2 < kMinTileLog2 ||
        c.tile_log2 > kMaxTileLog2 || (k.block != 256 && k.block != 512))
      continue;
    m[k] = c;
  }
  return m;
}

void append_tune_file(const char* path, const std::vector<std::pair<TuneKey, Choice>>& rows)
{
  if (!path || !*path || rows.empty()) return;
  std::ofstream f(path, std::ios::app);
  if (!f) return;  // a read-only location only loses the persistence
  for (auto& r : rows)
    f << r.first.device << ' ' << r.first.sig << ' ' << r.first.block << ' ' << r.first.cls << ' ' << r.second.mode
      << ' ' << r.second.smul << ' ' << r.second.tile_log2 << ' ' << static_cast<long long>(r.second.rate) << '\n';
}

// Remembered per device: cudaGetDeviceProperties costs milliseconds.
std::string device_tag(int device)
{
  static std::mutex mu;
  static std::map<int, std::string> known;
  std::lock_guard<std::mutex> lk(mu);
  auto it = known.find(device);
  if (it != known.end()) return it->second;
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
  std::string s = p.name;
  for (auto& ch : s)
    if (ch == ' ' || ch == '\t') ch = '_';
  char buf[64];
  snprintf(buf, sizeof(buf), "_sm%d%d_%d", p.major, p.minor, p.multiProcessorCount);
  return known[device] = s + buf;
}

// What the kernels' cost depends on: key words and accumulators per channel.
std::string schema_signature(const Plan& p)
{
  std::ostringstream os;
  os << "w" << p.key.nwords << "k" << p.key.ncols << (p.key.skip_null_rows ? "x" : "");
  for (int c = 0; c < p.nchan; ++c) {
    const Channel& ch = p.chan[c];
    os << "_c" << int(ch.ptype) << "n" << std::hex << ch.need << std::dec << (ch.a_cnt >= 0 ? "m" : "")
       << (ch.idx_width ? "d" : "");
  }
  return os.str();
}

}  // namespace
}  // namespace gbx

// --------------------------------------------------------------- the batch

struct gbx_batch {
  // schema (instance 0's types, nullability of all instances)
  Plan schema{};
  int32_t null_policy = GBX_NULL_EXCLUDE;
  int nkeys           = 0;
  int nreq            = 0;
  std::vector<int> req_chan;
  std::vector<gbx_column_view> key_types;   // type_id / scale of each key column
  std::vector<gbx_column_view> req_values;  // request q's value column of instance 0 (types only)
  std::vector<std::vector<gbx_aggregation>> req_aggs;
  std::vector<int64_t> chan_nullable;       // 1 when any instance's channel may hold nulls

  // per instance
  struct Inst {
    int64_t n    = 0;
    double est   = 1;
    int cls      = 0;
    int32_t mode = BM_GLOBAL;
    uint32_t S   = 0;  // shared-memory slots
    uint64_t cap = 0;  // global table slots
    int64_t tile = 0;
    InstCols cols{};
  };
  std::vector<Inst> inst;

  gbx::DeviceInfo dev;
  gbx::Alloc alloc;
  cudaStream_t cs = nullptr;  // capture / housekeeping stream
  bool one_shot   = false;    // no graph: execute issues the kernels itself
  int block       = 256;
  size_t smem     = 0;
  int grid        = 0;

  // device state (rebuilt on a re-plan)
  std::vector<std::pair<void*, size_t>> dbufs;
  BatchInst* d_inst   = nullptr;
  BatchItem* d_items  = nullptr;
  uint32_t nitems     = 0;
  uint32_t* d_counter = nullptr;
  int32_t* d_status   = nullptr;
  uint32_t* d_special = nullptr;
  int64_t* d_counts   = nullptr;
  int64_t* d_offsets  = nullptr;
  void* d_scan_temp   = nullptr;
  size_t scan_bytes   = 0;
  unsigned long long* d_nulls = nullptr;
  int64_t out_rows   = 0;
  size_t arena_bytes = 0;
  std::vector<BatchInst> h_inst;
  OutPlan op{};
  std::vector<gbx_column> key_cols;
  std::vector<std::vector<gbx_column>> res_cols;
  std::vector<gbx_aggregation_result> res_reqs;
  cudaGraph_t graph    = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2]    = {nullptr, nullptr};                    // around the launch
  cudaEvent_t phase[4] = {nullptr, nullptr, nullptr, nullptr};  // recorded by the execution itself

  // host copies written by each execution: pinned for a captured graph,
  // pageable for a one-shot batch (pinned allocation and release synchronise
  // with the whole device, which would stall every other stream's work)
  int64_t* h_offsets          = nullptr;
  int32_t* h_status           = nullptr;
  unsigned long long* h_nulls = nullptr;
  bool pinned_host            = true;
  bool owns_stream            = true;  // a one-shot batch runs on the caller's stream

  gbx_batch_output output{};
  gbx_batch_stats stats{};

  void* dalloc(size_t bytes)
  {
    void* p = alloc.allocate(bytes);
    dbufs.emplace_back(p, bytes);
    return p;
  }

  void release_device()
  {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec     = nullptr;
    graph    = nullptr;
    alloc.st = cs;
    for (auto& b : dbufs) alloc.release(b.first, b.second);
    dbufs.clear();
    if (cs) cudaStreamSynchronize(cs);
    key_cols.clear();
    res_cols.clear();
    res_reqs.clear();
  }

  ~gbx_batch()
  {
    release_device();
    if (pinned_host) {
      if (h_offsets) cudaFreeHost(h_offsets);
      if (h_status) cudaFreeHost(h_status);
      if (h_nulls) cudaFreeHost(h_nulls);
    } else {
      delete[] h_offsets;
      delete[] h_status;
      delete[] h_nulls;
    }
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : phase)
      if (e) cudaEventDestroy(e);
    if (cs && owns_stream) cudaStreamDestroy(cs);
  }
};

namespace gbx {
namespace {

int64_t maybe_nulls(const gbx_column_view& c) { return (c.null_mask != nullptr && c.null_count != 0) ? 1 : 0; }

// The instance's buffers in kernel form.
InstCols inst_cols(const gbx_batch& b, const gbx_batch_instance& in)
{
  InstCols ic{};
  for (int c = 0; c < b.nkeys; ++c) {
    const gbx_column_view& k = in.keys.columns[c];
    ic.key[c].data           = k.data;
    ic.key[c].mask           = maybe_nulls(k) ? k.null_mask : nullptr;
    ic.key[c].offset         = k.offset;
  }
  std::vector<int> rc;
  std::vector<const gbx_column_view*> chans = collect_channels(in.requests, b.nreq, rc);
  for (size_t c = 0; c < chans.size(); ++c) {
    const gbx_column_view& v = *chans[c];
    InstChan& ch             = ic.chan[c];
    ch.data                  = v.data;
    ch.mask                  = maybe_nulls(v) ? v.null_mask : nullptr;
    ch.offset                = v.offset;
    if (v.type_id == GBX_TYPE_DICTIONARY32) {
      ch.dict_data   = v.dict_keys->data;
      ch.dict_offset = v.dict_keys->offset;
      ch.dict_size   = v.dict_keys->size;
    }
  }
  return ic;
}

bool same_value_shape(const gbx_column_view& a, const gbx_column_view& b)
{
  if (a.type_id != b.type_id || a.scale != b.scale) return false;
  if (a.type_id == GBX_TYPE_DICTIONARY32) {
    int32_t ia = a.index_type_id ? a.index_type_id : GBX_TYPE_INT32;
    int32_t ib = b.index_type_id ? b.index_type_id : GBX_TYPE_INT32;
    if (ia != ib || !a.dict_keys || !b.dict_keys) return false;
    if (a.dict_keys->type_id != b.dict_keys->type_id || a.dict_keys->scale != b.dict_keys->scale) return false;
  }
  return true;
}

// Checks that every instance follows instance 0's schema and builds the
// schema plan (nullability: any instance's).  Host only.
void build_schema(gbx_batch& b, const gbx_batch_instance* ins, int32_t ninst)
{
  const gbx_batch_instance& i0 = ins[0];
  GBX_EXPECTS(i0.keys.num_columns >= 1 && i0.keys.columns != nullptr, "a batch instance needs key columns");
  b.nkeys = i0.keys.num_columns;
  GBX_EXPECTS(b.nkeys <= kMaxKeyCols, "more than %d key columns", kMaxKeyCols);
  b.key_types.assign(i0.keys.columns, i0.keys.columns + b.nkeys);
  for (auto& k : b.key_types) {
    if (k.type_id == GBX_TYPE_DICTIONARY32)
      fail(GBX_ERR_UNSUPPORTED, "dictionary key columns are not supported in a batch (instances would not share "
                                "one dictionary); decode them or use gbx_groupby_aggregate");
    if (!is_fixed_width(k.type_id))
      fail(GBX_ERR_UNSUPPORTED, "key type %d (string / list / struct / decimal128) is not supported by this library",
           k.type_id);
  }
  GBX_EXPECTS(b.nreq == 0 || i0.requests != nullptr, "batch instance 0 has no requests");
  std::vector<const gbx_column_view*> chan0 = collect_channels(i0.requests, b.nreq, b.req_chan);
  b.req_values.clear();
  b.req_aggs.clear();
  for (int q = 0; q < b.nreq; ++q) {
    b.req_values.push_back(i0.requests[q].values);
    b.req_aggs.emplace_back(i0.requests[q].aggregations, i0.requests[q].aggregations + i0.requests[q].num_aggregations);
  }
  std::vector<int64_t> key_null(b.nkeys, 0);
  b.chan_nullable.assign(chan0.size(), 0);
  for (int32_t i = 0; i < ninst; ++i) {
    const gbx_batch_instance& in = ins[i];
    GBX_EXPECTS(in.keys.num_columns == b.nkeys && in.keys.columns != nullptr,
                "batch instance %d has %d key columns, instance 0 has %d", i, in.keys.num_columns, b.nkeys);
    const int64_t n = in.keys.columns[0].size;
    GBX_EXPECTS(n >= 0 && n <= INT32_MAX, "batch instance %d: row count out of range", i);
    for (int c = 0; c < b.nkeys; ++c) {
      const gbx_column_view& k = in.keys.columns[c];
      GBX_EXPECTS(k.type_id == b.key_types[c].type_id && k.scale == b.key_types[c].scale,
                  "batch instance %d: key column %d differs in type from instance 0", i, c);
      GBX_EXPECTS(k.size == n, "batch instance %d: key columns differ in size", i);
      GBX_EXPECTS(k.offset >= 0, "negative offset");
      key_null[c] |= maybe_nulls(k);
    }
    GBX_EXPECTS(b.nreq == 0 || in.requests != nullptr, "batch instance %d has no requests", i);
    validate_requests(in.requests, b.nreq, n);
    // ARGMIN / ARGMAX index rows of the caller's column (the batched kernels
    // address rows within their instance); M2 and the kinds that sort a
    // group's values are computed by gbx_groupby_aggregate only
    for (int q = 0; q < b.nreq; ++q)
      for (int k = 0; k < in.requests[q].num_aggregations; ++k) {
        const int32_t kind = in.requests[q].aggregations[k].kind;
        if (!is_batch_kind(kind))
          fail(GBX_ERR_UNSUPPORTED, "aggregation kind %d is not provided by the batched form; use gbx_groupby_aggregate",
               kind);
      }
    std::vector<int> rc;
    std::vector<const gbx_column_view*> chans = collect_channels(in.requests, b.nreq, rc);
    GBX_EXPECTS(rc == b.req_chan, "batch instance %d shares value columns between requests differently from instance 0",
                i);
    for (int q = 0; q < b.nreq; ++q) {
      const gbx_request& r = in.requests[q];
      GBX_EXPECTS(same_value_shape(r.values, b.req_values[q]), "batch instance %d: request %d's values differ in type",
                  i, q);
      GBX_EXPECTS(r.num_aggregations == static_cast<int32_t>(b.req_aggs[q].size()),
                  "batch instance %d: request %d differs in aggregations", i, q);
      for (int k = 0; k < r.num_aggregations; ++k)
        GBX_EXPECTS(r.aggregations[k].kind == b.req_aggs[q][k].kind && r.aggregations[k].ddof == b.req_aggs[q][k].ddof,
                    "batch instance %d: request %d differs in aggregations", i, q);
    }
    for (size_t c = 0; c < chans.size(); ++c) b.chan_nullable[c] |= maybe_nulls(*chans[c]);
  }
  bool ok      = true;
  b.schema.key = make_key_plan(i0.keys.columns, b.nkeys, b.null_policy, key_null, ok);
  if (!ok) fail(GBX_ERR_UNSUPPORTED, "key columns need more than 128 packed bits; wider composite keys are not supported");
  fill_channels(b.schema, chan0, b.chan_nullable, i0.requests, b.nreq, b.req_chan);
  // the buffers come from each instance's InstCols
  for (int c = 0; c < b.schema.key.ncols; ++c) {
    b.schema.key.cols[c].data = nullptr;
    b.schema.key.cols[c].mask = nullptr;
  }
  for (int c = 0; c < b.schema.nchan; ++c) {
    b.schema.chan[c].data      = nullptr;
    b.schema.chan[c].mask      = nullptr;
    b.schema.chan[c].dict_data = nullptr;
    b.schema.chan[c].dict_size = 0;
  }
  int nout = 0;
  for (auto& a : b.req_aggs) nout += static_cast<int>(a.size());
  if (nout > kMaxOut) fail(GBX_ERR_UNSUPPORTED, "more than %d results in one call", kMaxOut);
}

// Table slots and shared-memory needs of one instance under its choice.
void apply_choice(gbx_batch& b, gbx_batch::Inst& I, const Choice& c, int64_t tile_override)
{
  I.mode = c.mode;
  I.S    = 0;
  if (c.mode == BM_SHARED || c.mode == BM_WARP) {
    uint32_t S        = base_slots(I.cls) << c.smul;
    const size_t need = (c.mode == BM_WARP ? b.block / 32 : 1) * static_cast<size_t>(make_smem_layout(b.schema, S).total);
    if (need > smem_budget(b.block)) I.mode = BM_GLOBAL;
    else I.S = S;
  }
  I.tile = tile_override > 0 ? tile_override : (int64_t(1) << c.tile_log2);
  // global table at load <= ~0.4 of the estimate (room for its error);
  // never more slots than rows need
  const uint64_t want = next_pow2(static_cast<uint64_t>(std::max(64.0, std::ceil(I.est * 2.5))));
  I.cap = std::min<uint64_t>(want, next_pow2(2 * static_cast<uint64_t>(I.n) + 2));
  I.cap = std::max<uint64_t>(I.cap, 64);
}

Choice default_choice(const gbx_batch& b, int cls)
{
  // without measurements: a CTA-shared table when it fits, else the global table
  Choice c;
  c.tile_log2 = 16;
  for (int smul = 1; smul >= 0; --smul) {
    const uint32_t S = base_slots(cls) << smul;
    if (make_smem_layout(b.schema, S).total <= smem_budget(b.block)) {
      c.mode = BM_SHARED;
      c.smul = smul;
      return c;
    }
  }
  c.mode = BM_GLOBAL;
  return c;
}

// Every operation of one execution, in stream order: clears, table fill, the
// persistent aggregation, counting + offsets, output writing, and the copies
// of offsets, statuses and null counts to pinned host memory.
cudaError_t enqueue_batch(gbx_batch& b, cudaStream_t s)
{
  const int ninst = static_cast<int>(b.inst.size());
  cudaError_t err = cudaSuccess;
  auto step       = [&](cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  };
  // under capture an event record must be an external node to be recorded
  // when the graph runs (a plain record only orders the capture)
  const unsigned rec_flags = b.one_shot ? cudaEventRecordDefault : cudaEventRecordExternal;
  auto mark                = [&](cudaEvent_t e) { step(cudaEventRecordWithFlags(e, s, rec_flags)); };
  step(cudaMemsetAsync(b.d_counter, 0, 16, s));
  step(cudaMemsetAsync(b.d_nulls, 0, (kMaxKeyCols + kMaxOut) * 8, s));
  for (auto& c : b.key_cols)
    if (c.null_mask) step(cudaMemsetAsync(c.null_mask, 0, c.mask_bytes, s));
  for (auto& q : b.res_cols)
    for (auto& c : q)
      if (c.null_mask) step(cudaMemsetAsync(c.null_mask, 0, c.mask_bytes, s));
  mark(b.phase[0]);
  step(launch_batch_init(b.schema, b.d_inst, ninst, s));
  mark(b.phase[1]);
  step(launch_batch_agg(b.schema, b.d_inst, b.d_items, b.nitems, b.d_counter, b.block, b.grid, b.smem, s));
  mark(b.phase[2]);
  step(launch_batch_count(b.schema, b.d_inst, ninst, b.d_counts, b.d_offsets, b.d_scan_temp, &b.scan_bytes, s));
  step(launch_batch_write(b.schema, b.d_inst, ninst, b.d_offsets, b.op, s));
  mark(b.phase[3]);
  step(cudaMemcpyAsync(b.h_offsets, b.d_offsets, (static_cast<size_t>(ninst) + 1) * 8, cudaMemcpyDeviceToHost, s));
  step(cudaMemcpyAsync(b.h_status, b.d_status, static_cast<size_t>(ninst) * 4, cudaMemcpyDeviceToHost, s));
  step(cudaMemcpyAsync(b.h_nulls, b.d_nulls, (kMaxKeyCols + kMaxOut) * 8, cudaMemcpyDeviceToHost, s));
  return err;
}

// Arena, descriptors, work items, outputs (sized for every instance's bound)
// and the graph.  `with_outputs` false builds what the tuner's timing needs.
void build_device(gbx_batch& b, bool with_outputs)
{
  b.release_device();
  const int ninst     = static_cast<int>(b.inst.size());
  const size_t sbytes = slot_bytes(b.schema);
  cudaStream_t s      = b.cs;
  b.alloc.st          = s;

  // ---- arena: one region per instance, 8-byte arrays first
  std::vector<size_t> region(ninst);
  size_t arena = 0;
  for (int i = 0; i < ninst; ++i) {
    region[i] = arena;
    arena += ((b.inst[i].cap + 1) * sbytes + 255) & ~size_t(255);
  }
  b.arena_bytes = arena;
  char* base    = static_cast<char*>(b.dalloc(arena));
  b.d_status    = static_cast<int32_t*>(b.dalloc(static_cast<size_t>(ninst) * 4));
  b.d_special   = static_cast<uint32_t*>(b.dalloc(static_cast<size_t>(ninst) * 4));
  b.d_counter   = static_cast<uint32_t*>(b.dalloc(16));
  b.h_inst.assign(ninst, BatchInst{});
  size_t smem_need = 0;
  for (int i = 0; i < ninst; ++i) {
    const gbx_batch::Inst& I = b.inst[i];
    BatchInst& D             = b.h_inst[i];
    D.cols                   = I.cols;
    D.num_rows               = I.n;
    D.mode                   = I.mode;
    TableRef& t              = D.t;
    t.cap                    = I.cap;
    char* p                  = base + region[i];
    const size_t slots       = I.cap + 1;
    t.keys                   = reinterpret_cast<uint64_t*>(p);
    p += slots * b.schema.key.nwords * 8;
    for (int a = 0; a < b.schema.acc.nacc; ++a)
      if (acc_bytes(b.schema.acc.kind[a]) == 8) {
        t.acc[a] = p;
        p += slots * 8;
      }
    for (int a = 0; a < b.schema.acc.nacc; ++a)
      if (acc_bytes(b.schema.acc.kind[a]) == 4) {
        t.acc[a] = p;
        p += slots * 4;
      }
    t.rows         = reinterpret_cast<uint32_t*>(p);
    t.special_used = b.d_special + i;
    t.status       = b.d_status + i;
    if (I.mode == BM_SHARED || I.mode == BM_WARP) {
      D.sl              = make_smem_layout(b.schema, I.S);
      const size_t need = (I.mode == BM_WARP ? b.block / 32 : 1) * static_cast<size_t>(D.sl.total);
      smem_need         = std::max(smem_need, need);
    }
  }
  b.smem = smem_need;
  GBX_CUDA(batch_agg_max_grid(b.schema, b.block, b.smem, b.dev.num_sms, &b.grid));

  // ---- work items, largest first
  std::vector<BatchItem> items;
  for (int i = 0; i < ninst; ++i) {
    const int64_t n = b.inst[i].n, tile = std::max<int64_t>(b.inst[i].tile, 1024);
    for (int64_t r = 0; r < n; r += tile) items.push_back(BatchItem{static_cast<uint32_t>(i), 0u, r, std::min(n, r + tile)});
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const BatchItem& x, const BatchItem& y) { return (x.end - x.begin) > (y.end - y.begin); });
  b.nitems  = static_cast<uint32_t>(items.size());
  b.d_inst  = static_cast<BatchInst*>(b.dalloc(static_cast<size_t>(ninst) * sizeof(BatchInst)));
  b.d_items = static_cast<BatchItem*>(b.dalloc(std::max<size_t>(1, items.size()) * sizeof(BatchItem)));
  GBX_CUDA(cudaMemcpyAsync(b.d_inst, b.h_inst.data(), static_cast<size_t>(ninst) * sizeof(BatchInst),
                           cudaMemcpyHostToDevice, s));
  if (!items.empty())
    GBX_CUDA(cudaMemcpyAsync(b.d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
  GBX_CUDA(cudaStreamSynchronize(s));  // `items` is host memory of this frame
  if (!with_outputs) return;

  // ---- outputs: every instance has at most min(rows, cap + 1) groups
  int64_t rows = 0;
  for (auto& I : b.inst) rows += std::min<int64_t>(I.n, static_cast<int64_t>(I.cap) + 1);
  b.out_rows = rows;
  b.op       = OutPlan{};
  b.key_cols.assign(b.nkeys, gbx_column{});
  for (int c = 0; c < b.nkeys; ++c) {
    const bool with_mask = b.schema.key.cols[c].null_bit != 0;
    alloc_column(b.alloc, b.key_cols[c], b.key_types[c].type_id, b.key_types[c].scale, rows, with_mask);
    b.dbufs.emplace_back(b.key_cols[c].data, b.key_cols[c].data_bytes);
    if (b.key_cols[c].null_mask) b.dbufs.emplace_back(b.key_cols[c].null_mask, b.key_cols[c].mask_bytes);
    b.op.key_data[c] = b.key_cols[c].data;
    b.op.key_mask[c] = b.key_cols[c].null_mask;
  }
  b.res_cols.assign(b.nreq, {});
  for (int q = 0; q < b.nreq; ++q) {
    const gbx_column_view& v = b.req_values[q];
    const int32_t vt         = value_type(v);
    for (size_t k = 0; k < b.req_aggs[q].size(); ++k) {
      const int32_t kind   = b.req_aggs[q][k].kind;
      const int32_t tt     = target_type(vt, kind);
      const bool has_nulls = b.chan_nullable[b.req_chan[q]] != 0;
      // nullable iff the values may hold nulls; COUNT never; VAR/STD always (hash/groupby.cu:424-454)
      const bool with_mask = (kind == GBX_AGG_COUNT_VALID || kind == GBX_AGG_COUNT_ALL)
                               ? false
                               : (has_nulls || kind == GBX_AGG_VARIANCE || kind == GBX_AGG_STD);
      const int32_t scale  = is_decimal(tt) ? (v.type_id == GBX_TYPE_DICTIONARY32 ? v.dict_keys->scale : v.scale) : 0;
      gbx_column col{};
      alloc_column(b.alloc, col, tt, scale, rows, with_mask);
      b.dbufs.emplace_back(col.data, col.data_bytes);
      if (col.null_mask) b.dbufs.emplace_back(col.null_mask, col.mask_bytes);
      OutCol& o   = b.op.out[b.op.nout++];
      o.data      = col.data;
      o.mask      = col.null_mask;
      o.kind      = kind;
      o.ddof      = b.req_aggs[q][k].ddof;
      o.chan      = static_cast<int8_t>(b.req_chan[q]);
      o.out_ptype = phys_of(tt);
      o.out_width = static_cast<int8_t>(type_width(tt));
      b.res_cols[q].push_back(col);
    }
  }
  b.d_nulls        = static_cast<unsigned long long*>(b.dalloc((kMaxKeyCols + kMaxOut) * 8));
  b.op.null_counts = b.d_nulls;
  b.d_counts       = static_cast<int64_t*>(b.dalloc((static_cast<size_t>(ninst) + 1) * 8));
  b.d_offsets      = static_cast<int64_t*>(b.dalloc((static_cast<size_t>(ninst) + 1) * 8));
  b.scan_bytes     = 0;
  GBX_CUDA(launch_batch_count(b.schema, b.d_inst, ninst, b.d_counts, b.d_offsets, nullptr, &b.scan_bytes, s));
  b.d_scan_temp = b.dalloc(std::max<size_t>(b.scan_bytes, 16));

  // ---- the graph (a one-shot batch issues the same sequence at execute)
  GBX_CUDA(cudaStreamSynchronize(s));
  if (b.one_shot) {
    b.stats.graph_nodes         = 0;
    b.stats.kernels_per_execute = 5;  // init, aggregate, count, scan, write
    return;
  }
  GBX_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = enqueue_batch(b, s);
  cudaGraph_t g   = nullptr;
  cudaError_t ec  = cudaStreamEndCapture(s, &g);
  if (err != cudaSuccess || ec != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    GBX_CUDA(err != cudaSuccess ? err : ec);
  }
  b.graph = g;
  GBX_CUDA(cudaGraphInstantiate(&b.exec, b.graph, 0));
  size_t nodes = 0;
  GBX_CUDA(cudaGraphGetNodes(b.graph, nullptr, &nodes));
  std::vector<cudaGraphNode_t> nv(nodes);
  GBX_CUDA(cudaGraphGetNodes(b.graph, nv.data(), &nodes));
  int kernels = 0;
  for (auto& nd : nv) {
    cudaGraphNodeType ty;
    GBX_CUDA(cudaGraphNodeGetType(nd, &ty));
    kernels += ty == cudaGraphNodeTypeKernel ? 1 : 0;
  }
  b.stats.graph_nodes         = static_cast<int32_t>(nodes);
  b.stats.kernels_per_execute = kernels;
}

// rows/s of the aggregation kernel over `subset` with every member on choice `c`.
double measure(const gbx_batch& b, const std::vector<int>& subset, int block, const Choice& c)
{
  gbx_batch t;
  t.schema      = b.schema;
  t.null_policy = b.null_policy;
  t.nkeys       = b.nkeys;
  t.nreq        = b.nreq;
  t.dev         = b.dev;
  t.alloc       = b.alloc;
  t.cs          = b.cs;  // borrowed: cleared before `t` goes away
  t.block       = block;
  int64_t rows  = 0;
  for (int i : subset) {
    t.inst.push_back(b.inst[i]);
    apply_choice(t, t.inst.back(), c, 0);
    rows += b.inst[i].n;
  }
  if (c.mode != BM_GLOBAL)
    for (auto& I : t.inst)
      if (I.mode == BM_GLOBAL) {
        t.cs = nullptr;  // the candidate does not fit this block shape
        return 0.0;
      }
  double best     = 0.0;
  cudaEvent_t e0  = nullptr, e1 = nullptr;
  try {
    build_device(t, false);
    GBX_CUDA(cudaEventCreate(&e0));
    GBX_CUDA(cudaEventCreate(&e1));
    float ms_min = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      GBX_CUDA(cudaMemsetAsync(t.d_counter, 0, 16, t.cs));
      GBX_CUDA(launch_batch_init(t.schema, t.d_inst, static_cast<int>(t.inst.size()), t.cs));
      GBX_CUDA(cudaEventRecord(e0, t.cs));
      GBX_CUDA(launch_batch_agg(t.schema, t.d_inst, t.d_items, t.nitems, t.d_counter, t.block, t.grid, t.smem, t.cs));
      GBX_CUDA(cudaEventRecord(e1, t.cs));
      GBX_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      GBX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0) ms_min = std::min(ms_min, ms);  // the first run warms up
    }
    std::vector<int32_t> st(t.inst.size());
    GBX_CUDA(cudaMemcpy(st.data(), t.d_status, st.size() * 4, cudaMemcpyDeviceToHost));
    bool clean = true;
    for (auto v : st) clean &= (v & (S_SPIN_LIMIT | S_BAD_INDEX)) == 0;
    best = clean ? static_cast<double>(rows) / (ms_min * 1e-3) : 0.0;
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    t.release_device();
    t.cs = nullptr;
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  t.release_device();
  t.cs = nullptr;
  return best;
}

// Chooses a block shape and, per tuning class, mode / table / tile.
void plan_batch(gbx_batch& b, const gbx_batch_options& o)
{
  const auto t0 = std::chrono::steady_clock::now();
  std::map<int, std::vector<int>> classes;
  std::map<int, int64_t> class_rows;
  for (int i = 0; i < static_cast<int>(b.inst.size()); ++i) {
    classes[b.inst[i].cls].push_back(i);
    class_rows[b.inst[i].cls] += b.inst[i].n;
  }
  b.stats.classes          = static_cast<int32_t>(classes.size());
  const std::string device = o.tune != GBX_TUNE_OFF ? device_tag(b.dev.device) : std::string();
  const std::string sig    = schema_signature(b.schema);
  std::map<TuneKey, Choice> table;
  if (o.tune != GBX_TUNE_OFF) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    table = read_tune_file(o.tune_file);
  }
  std::vector<std::pair<TuneKey, Choice>> fresh;
  const std::vector<int> blocks = o.block_threads ? std::vector<int>{o.block_threads} : std::vector<int>{256, 512};
  std::map<int, std::map<int, Choice>> chosen;  // block -> class -> choice
  int measured = 0, cached = 0;
  for (int blk : blocks) {
    b.block = blk;
    for (auto& kv : classes) {
      const int cls = kv.first;
      TuneKey key{device, sig, blk, cls};
      auto it         = table.find(key);
      const bool have = it != table.end() && it->second.rate > 0;
      if (o.tune == GBX_TUNE_ALL || (o.tune == GBX_TUNE_MISSING && !have)) {
        // representatives: the class's largest instances, up to ~16M rows
        std::vector<int> members = kv.second;
        std::stable_sort(members.begin(), members.end(), [&](int x, int y) { return b.inst[x].n > b.inst[y].n; });
        std::vector<int> subset;
        int64_t rows = 0;
        for (int i : members) {
          if (subset.size() >= 64 || rows >= (int64_t(16) << 20)) break;
          subset.push_back(i);
          rows += b.inst[i].n;
        }
        std::vector<Choice> cand;
        for (int tl : {15, 17}) {
          for (int smul = 0; smul <= 1; ++smul) {
            Choice c;
            c.mode = BM_SHARED, c.smul = smul, c.tile_log2 = tl;
            cand.push_back(c);
          }
          Choice w;
          w.mode = BM_WARP, w.smul = 0, w.tile_log2 = tl;
          cand.push_back(w);
          Choice g;
          g.mode = BM_GLOBAL, g.tile_log2 = tl;
          cand.push_back(g);
        }
        Choice best;
        best.rate = -1;
        for (Choice c : cand) {
          c.rate = measure(b, subset, blk, c);
          if (c.rate > best.rate) best = c;
        }
        if (best.rate <= 0) best = default_choice(b, cls);
        chosen[blk][cls] = best;
        fresh.emplace_back(key, best);
        ++measured;
      } else if (have && o.tune != GBX_TUNE_OFF) {
        chosen[blk][cls] = it->second;
        ++cached;
      } else {
        chosen[blk][cls] = default_choice(b, cls);
      }
    }
  }
  // block shape: the least predicted time, among shapes whose every class has a rate
  int best_blk = blocks[0];
  if (blocks.size() > 1) {
    double best_t = -1;
    for (int blk : blocks) {
      double tsum = 0;
      bool all    = true;
      for (auto& kv : chosen[blk]) {
        if (kv.second.rate <= 0) {
          all = false;
          break;
        }
        tsum += static_cast<double>(class_rows[kv.first]) / kv.second.rate;
      }
      if (!all) continue;
      if (best_t < 0 || tsum < best_t) {
        best_t   = tsum;
        best_blk = blk;
      }
    }
  }
  b.block = best_blk;
  for (auto& I : b.inst) {
    Choice c = chosen[best_blk][I.cls];
    if (o.force_mode != GBX_BATCH_MODE_AUTO) {
      c.mode = o.force_mode;
      c.smul = 0;
    }
    apply_choice(b, I, c, o.tile_rows);
  }
  if (!fresh.empty()) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    append_tune_file(o.tune_file, fresh);
  }
  b.stats.classes_measured = measured;
  b.stats.classes_cached   = cached;
  b.stats.tune_ms =
    measured ? std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count() : 0.0f;
}

}  // namespace
}  // namespace gbx

// ================================================================== C ABI

extern "C" {

int gbx_batch_create(const gbx_batch_instance* instances, int32_t num_instances, int32_t num_requests,
                     const gbx_batch_options* options, void* stream, const gbx_allocator* mr, gbx_batch** out)
{
  gbx_batch* b = nullptr;
  int st       = guarded([&] {
    const auto t0 = std::chrono::steady_clock::now();
    GBX_EXPECTS(out != nullptr, "out is null");
    *out = nullptr;
    GBX_EXPECTS(instances != nullptr && num_instances >= 1, "a batch needs at least one instance");
    GBX_EXPECTS(num_requests >= 0, "negative request count");
    gbx_batch_options o{};
    if (options) o = *options;
    GBX_EXPECTS(o.null_policy == GBX_NULL_EXCLUDE || o.null_policy == GBX_NULL_INCLUDE, "invalid null_policy");
    GBX_EXPECTS(o.tune >= GBX_TUNE_OFF && o.tune <= GBX_TUNE_ALL, "invalid tune setting");
    GBX_EXPECTS(o.force_mode >= GBX_BATCH_MODE_AUTO && o.force_mode <= GBX_BATCH_MODE_GLOBAL, "invalid force_mode");
    GBX_EXPECTS(o.block_threads == 0 || o.block_threads == 256 || o.block_threads == 512,
                "block_threads must be 0, 256 or 512");
    GBX_EXPECTS(o.tile_rows >= 0, "negative tile_rows");

    b              = new gbx_batch();
    b->null_policy = o.null_policy;
    b->nreq        = num_requests;
    b->one_shot    = o.one_shot != 0;
    if (mr && mr->allocate && mr->deallocate) {
      b->alloc.user     = *mr;
      b->alloc.has_user = true;
    }
    build_schema(*b, instances, num_instances);  // host-only checks first
    b->dev = current_device();
    if (b->one_shot) {
      // no graph to capture: the caller's stream orders everything, and the
      // host copies need not be pinned
      b->cs          = static_cast<cudaStream_t>(stream);
      b->owns_stream = false;
      b->pinned_host = false;
      b->h_offsets   = new int64_t[static_cast<size_t>(num_instances) + 1];
      b->h_status    = new int32_t[static_cast<size_t>(num_instances)];
      b->h_nulls     = new unsigned long long[kMaxKeyCols + kMaxOut];
    } else {
      GBX_CUDA(cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking));
      // the caller's stream may still be producing the inputs
      cudaEvent_t ready;
      GBX_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
      GBX_CUDA(cudaEventRecord(ready, static_cast<cudaStream_t>(stream)));
      GBX_CUDA(cudaStreamWaitEvent(b->cs, ready, 0));
      cudaEventDestroy(ready);
      GBX_CUDA(cudaMallocHost(&b->h_offsets, (static_cast<size_t>(num_instances) + 1) * 8));
      GBX_CUDA(cudaMallocHost(&b->h_status, static_cast<size_t>(num_instances) * 4));
      GBX_CUDA(cudaMallocHost(&b->h_nulls, (kMaxKeyCols + kMaxOut) * 8));
    }
    b->alloc.st = b->cs;
    for (auto& e : b->ev) GBX_CUDA(cudaEventCreate(&e));
    for (auto& e : b->phase) GBX_CUDA(cudaEventCreate(&e));

    b->inst.resize(num_instances);
    for (int i = 0; i < num_instances; ++i) {
      b->inst[i].n    = instances[i].keys.columns[0].size;
      b->inst[i].cols = inst_cols(*b, instances[i]);
    }
    // ---- sampled distinct count per instance
    {
      std::vector<BatchInst> h(num_instances);
      for (int i = 0; i < num_instances; ++i) {
        h[i].cols     = b->inst[i].cols;
        h[i].num_rows = b->inst[i].n;
      }
      auto* d    = static_cast<BatchInst*>(b->alloc.allocate(h.size() * sizeof(BatchInst)));
      auto* dout = static_cast<uint32_t*>(b->alloc.allocate(static_cast<size_t>(num_instances) * 8));
      std::vector<uint32_t> hs(static_cast<size_t>(num_instances) * 2);
      cudaError_t e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(BatchInst), cudaMemcpyHostToDevice, b->cs);
      if (e == cudaSuccess) e = launch_batch_sample(b->schema, d, num_instances, kSamplePerInstance, dout, b->cs);
      if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), dout, hs.size() * 4, cudaMemcpyDeviceToHost, b->cs);
      if (e == cudaSuccess) e = cudaStreamSynchronize(b->cs);
      b->alloc.release(d, h.size() * sizeof(BatchInst));
      b->alloc.release(dout, static_cast<size_t>(num_instances) * 8);
      GBX_CUDA(e);
      for (int i = 0; i < num_instances; ++i) {
        auto& I         = b->inst[i];
        const int64_t m = std::min<int64_t>(I.n, kSamplePerInstance);
        I.est           = I.n == 0 ? 1.0 : estimate_groups(hs[2 * i], hs[2 * i + 1], I.n, m);
        I.cls           = class_of(I.est);
      }
    }
    plan_batch(*b, o);
    build_device(*b, true);
    b->stats.num_instances = num_instances;
    for (auto& I : b->inst) {
      b->stats.num_rows += I.n;
      b->stats.mode_count[I.mode] += 1;
    }
    b->stats.block_threads = b->block;
    b->stats.grid          = b->grid;
    b->stats.work_items    = static_cast<int32_t>(b->nitems);
    b->stats.dynamic_smem  = static_cast<int64_t>(b->smem);
    b->stats.arena_bytes   = static_cast<int64_t>(b->arena_bytes);
    b->stats.output_rows   = b->out_rows;
    b->stats.create_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out               = b;
  });
  if (st != GBX_OK) delete b;
  return st;
}

int gbx_batch_execute(gbx_batch* b, void* stream, const gbx_batch_output** out)
{
  return guarded([&] {
    GBX_EXPECTS(b != nullptr && out != nullptr, "null argument");
    *out            = nullptr;
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    const int ninst = static_cast<int>(b->inst.size());
    for (int attempt = 0;; ++attempt) {
      GBX_CUDA(cudaEventRecord(b->ev[0], s));
      if (b->one_shot) GBX_CUDA(enqueue_batch(*b, s));
      else GBX_CUDA(cudaGraphLaunch(b->exec, s));
      GBX_CUDA(cudaEventRecord(b->ev[1], s));
      GBX_CUDA(cudaStreamSynchronize(s));
      int32_t all = 0;
      std::vector<int> full;
      for (int i = 0; i < ninst; ++i) {
        all |= b->h_status[i];
        if (b->h_status[i] & S_TABLE_FULL) full.push_back(i);
      }
      if (all & S_SPIN_LIMIT) fail(GBX_ERR_DEVICE, "a bounded device loop gave up (status 0x%x)", all);
      if (all & S_BAD_INDEX) fail(GBX_ERR_LOGIC, "dictionary index out of range");
      if (full.empty()) break;
      // an instance held more groups than its table: size it for its rows
      if (attempt >= 2) fail(GBX_ERR_DEVICE, "batch table overflow persists after re-planning");
      for (int i : full) {
        auto& I = b->inst[i];
        I.est   = static_cast<double>(I.n);
        I.cap   = next_pow2(2 * static_cast<uint64_t>(I.n) + 2);
      }
      b->stats.retries++;
      build_device(*b, true);
    }
    GBX_CUDA(cudaEventElapsedTime(&b->stats.execute_ms, b->ev[0], b->ev[1]));
    GBX_CUDA(cudaEventElapsedTime(&b->stats.init_ms, b->phase[0], b->phase[1]));
    GBX_CUDA(cudaEventElapsedTime(&b->stats.aggregate_ms, b->phase[1], b->phase[2]));
    GBX_CUDA(cudaEventElapsedTime(&b->stats.output_ms, b->phase[2], b->phase[3]));
    const int64_t G       = b->h_offsets[ninst];
    b->stats.num_groups   = G;
    b->stats.output_rows  = b->out_rows;
    b->stats.arena_bytes  = static_cast<int64_t>(b->arena_bytes);
    b->stats.work_items   = static_cast<int32_t>(b->nitems);

    for (int c = 0; c < b->nkeys; ++c) {
      gbx_column& col     = b->key_cols[c];
      col.view.size       = G;
      col.view.null_count = col.null_mask ? static_cast<int64_t>(b->h_nulls[c]) : 0;
    }
    int o = 0;
    b->res_reqs.assign(b->nreq, gbx_aggregation_result{});
    for (int q = 0; q < b->nreq; ++q) {
      for (auto& col : b->res_cols[q]) {
        col.view.size       = G;
        col.view.null_count = col.null_mask ? static_cast<int64_t>(b->h_nulls[kMaxKeyCols + o]) : 0;
        ++o;
      }
      b->res_reqs[q].num_results = static_cast<int32_t>(b->res_cols[q].size());
      b->res_reqs[q].results     = b->res_cols[q].data();
    }
    gbx_batch_output& os          = b->output;
    os                            = gbx_batch_output{};
    os.num_instances              = ninst;
    os.group_offsets              = b->h_offsets;
    os.device_group_offsets       = b->d_offsets;
    os.columns.num_groups         = G;
    os.columns.num_key_columns    = b->nkeys;
    os.columns.num_requests       = b->nreq;
    os.columns.keys               = b->key_cols.data();
    os.columns.requests           = b->res_reqs.data();
    os.columns.internal           = nullptr;
    *out                          = &os;
  });
}

int gbx_batch_rebind(gbx_batch* b, const gbx_batch_instance* instances, int32_t num_instances)
{
  return guarded([&] {
    GBX_EXPECTS(b != nullptr && instances != nullptr, "null argument");
    GBX_EXPECTS(num_instances == static_cast<int32_t>(b->inst.size()), "rebind needs the batch's %d instances",
                static_cast<int>(b->inst.size()));
    // the new buffers must fit the batch's schema: same types and
    // aggregations, and nulls only where the batch's plan has room for them
    gbx_batch probe;
    probe.null_policy = b->null_policy;
    probe.nreq        = b->nreq;
    build_schema(probe, instances, num_instances);
    bool same = probe.nkeys == b->nkeys && probe.req_chan == b->req_chan;
    for (int c = 0; same && c < b->nkeys; ++c)
      same = probe.key_types[c].type_id == b->key_types[c].type_id && probe.key_types[c].scale == b->key_types[c].scale;
    for (int q = 0; same && q < b->nreq; ++q) {
      same = same_value_shape(probe.req_values[q], b->req_values[q]) && probe.req_aggs[q].size() == b->req_aggs[q].size();
      for (size_t k = 0; same && k < b->req_aggs[q].size(); ++k)
        same = probe.req_aggs[q][k].kind == b->req_aggs[q][k].kind && probe.req_aggs[q][k].ddof == b->req_aggs[q][k].ddof;
    }
    GBX_EXPECTS(same, "rebind needs instances of the batch's schema");
    bool fits = probe.schema.key.skip_null_rows <= b->schema.key.skip_null_rows;
    for (int c = 0; c < b->nkeys; ++c) fits &= probe.schema.key.cols[c].null_bit <= b->schema.key.cols[c].null_bit;
    for (size_t c = 0; c < b->chan_nullable.size(); ++c) fits &= probe.chan_nullable[c] <= b->chan_nullable[c];
    GBX_EXPECTS(fits, "rebind: the new columns hold nulls where the batch's columns had none; create a new batch");
    for (int i = 0; i < num_instances; ++i)
      GBX_EXPECTS(instances[i].keys.columns[0].size == b->inst[i].n, "rebind instance %d: row count differs", i);
    for (int i = 0; i < num_instances; ++i) {
      b->inst[i].cols   = inst_cols(*b, instances[i]);
      b->h_inst[i].cols = b->inst[i].cols;
    }
    GBX_CUDA(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), b->h_inst.size() * sizeof(BatchInst),
                             cudaMemcpyHostToDevice, b->cs));
    GBX_CUDA(cudaStreamSynchronize(b->cs));
  });
}

int gbx_batch_instance_plan(const gbx_batch* b, int32_t* modes, int64_t* table_slots, int64_t* estimated_groups)
{
  return guarded([&] {
    GBX_EXPECTS(b != nullptr, "null batch");
    for (size_t i = 0; i < b->inst.size(); ++i) {
      if (modes) modes[i] = b->inst[i].mode;
      if (table_slots)
        table_slots[i] = b->inst[i].mode == BM_GLOBAL ? static_cast<int64_t>(b->inst[i].cap)
                                                      : static_cast<int64_t>(b->inst[i].S);
      if (estimated_groups) estimated_groups[i] = static_cast<int64_t>(b->inst[i].est);
    }
  });
}

int gbx_batch_last_stats(const gbx_batch* b, gbx_batch_stats* out)
{
  return guarded([&] {
    GBX_EXPECTS(b != nullptr && out != nullptr, "null argument");
    *out = b->stats;
  });
}

void gbx_batch_destroy(gbx_batch* b) { delete b; }

}  // extern "C"
