// groupby_facade_test.cpp -- the reference's groupby gtests, restated against
// the drop-in C++ API (include/cudf/groupby.hpp over libgbx).  Each case cites
// the reference test (cpp/tests/groupby/*.cpp) whose vectors it uses;
// results are sorted by key before comparing, as groupby_test_util.cpp:89-96
// does.  Prints one line per case and exits non-zero on any failure.
#include <cudf/groupby.hpp>
#include <cudf/join.hpp>
#include <cudf/stream_compaction.hpp>

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

namespace {

int g_failures = 0;
std::vector<void*> g_buffers;

#define CHECK(cond, ...)                                         \
  do {                                                           \
    if (!(cond)) {                                               \
      std::printf("    check failed: %s: ", #cond);              \
      std::printf(__VA_ARGS__);                                  \
      std::printf("\n");                                         \
      throw std::runtime_error("check failed");                  \
    }                                                            \
  } while (0)

void run(char const* name, std::function<void()> const& body)
{
  try {
    body();
    std::printf("PASS %s\n", name);
  } catch (std::exception const& e) {
    ++g_failures;
    std::printf("FAIL %s (%s)\n", name, e.what());
  }
}

template <typename T>
T* to_device(std::vector<T> const& h)
{
  void* p = nullptr;
  cudaMalloc(&p, std::max<size_t>(h.size() * sizeof(T), 8));
  if (!h.empty()) cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  g_buffers.push_back(p);
  return static_cast<T*>(p);
}

cudf::bitmask_type* mask_of(std::vector<int> const& valid)
{
  std::vector<uint32_t> words((valid.size() + 31) / 32 + 16, 0);
  for (size_t i = 0; i < valid.size(); ++i)
    if (valid[i]) words[i / 32] |= 1u << (i % 32);
  return to_device(words);
}

int null_count_of(std::vector<int> const& v) { return static_cast<int>(std::count(v.begin(), v.end(), 0)); }

template <typename T>
cudf::column_view col(cudf::type_id t, std::vector<T> const& v, std::vector<int> const& valid = {})
{
  return cudf::column_view(cudf::data_type{t}, static_cast<cudf::size_type>(v.size()), to_device(v),
                           valid.empty() ? nullptr : mask_of(valid), valid.empty() ? 0 : null_count_of(valid));
}

template <typename T>
std::vector<T> host_values(cudf::column_view const& c)
{
  std::vector<T> h(c.size());
  if (c.size()) cudaMemcpy(h.data(), c.data<T>(), c.size() * sizeof(T), cudaMemcpyDeviceToHost);
  return h;
}

std::vector<int> host_valid(cudf::column_view const& c)
{
  std::vector<int> v(c.size(), 1);
  if (!c.nullable() || c.size() == 0) return v;
  std::vector<uint32_t> w((c.size() + 31) / 32);
  cudaMemcpy(w.data(), c.null_mask(), w.size() * 4, cudaMemcpyDeviceToHost);
  for (int i = 0; i < c.size(); ++i) v[i] = (w[i / 32] >> (i % 32)) & 1;
  return v;
}

// Runs one aggregation and returns (keys, values, validity) sorted by key,
// null keys last.
template <typename K, typename R>
void run_single(cudf::column_view keys, cudf::column_view vals, std::unique_ptr<cudf::groupby_aggregation> agg,
                std::vector<K>& out_k, std::vector<int>& out_kv, std::vector<R>& out_v, std::vector<int>& out_vv,
                cudf::null_policy policy = cudf::null_policy::EXCLUDE)
{
  std::vector<cudf::groupby::aggregation_request> requests(1);
  requests[0].values = vals;
  requests[0].aggregations.push_back(std::move(agg));
  cudf::groupby::groupby gb(cudf::table_view({keys}), policy);
  auto result = gb.aggregate(requests);
  auto kview  = result.first->view().column(0);
  auto vview  = result.second[0].results[0]->view();
  auto k      = host_values<K>(kview);
  auto kv     = host_valid(kview);
  auto v      = host_values<R>(vview);
  auto vv     = host_valid(vview);
  std::vector<size_t> order(k.size());
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    if (kv[a] != kv[b]) return kv[a] > kv[b];
    return k[a] < k[b];
  });
  out_k.clear(); out_kv.clear(); out_v.clear(); out_vv.clear();
  for (auto i : order) {
    out_k.push_back(k[i]);
    out_kv.push_back(kv[i]);
    out_v.push_back(v[i]);
    out_vv.push_back(vv[i]);
  }
}

template <typename T>
void expect_equal(std::vector<T> const& got, std::vector<T> const& want, char const* what)
{
  CHECK(got.size() == want.size(), "%s: size %zu != %zu", what, got.size(), want.size());
  for (size_t i = 0; i < got.size(); ++i) CHECK(got[i] == want[i], "%s[%zu]", what, i);
}

void expect_near(std::vector<double> const& got, std::vector<double> const& want, std::vector<int> const& valid)
{
  CHECK(got.size() == want.size(), "size %zu != %zu", got.size(), want.size());
  for (size_t i = 0; i < got.size(); ++i) {
    if (!valid[i]) continue;
    CHECK(std::fabs(got[i] - want[i]) <= 1e-12 * std::max(1.0, std::fabs(want[i])), "value[%zu] %.17g vs %.17g", i,
          got[i], want[i]);
  }
}

using cudf::type_id;
const std::vector<int32_t> K10{1, 2, 3, 1, 2, 2, 1, 3, 3, 2};
const std::vector<int32_t> K11{1, 2, 3, 1, 2, 2, 1, 3, 3, 2, 4};
const std::vector<int> K11V{1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 1};

}  // namespace

int main()
{
  run("sum_tests.cpp:38-54 basic", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<int64_t> v;
    run_single(col(type_id::INT32, K10), col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9}),
               cudf::make_sum_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_equal(k, std::vector<int32_t>{1, 2, 3}, "keys");
    expect_equal(v, std::vector<int64_t>{9, 19, 17}, "sums");
  });
  run("keys_tests.cpp:199-225 pre_sorted_keys_nulls_before_include_nulls (sorted::YES, row order)", [] {
    std::vector<cudf::groupby::aggregation_request> requests(1);
    auto keys      = col(type_id::INT32, std::vector<int32_t>{1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4},
                         {1, 1, 1, 0, 0, 1, 1, 0, 1, 1, 1});
    auto vals      = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4});
    requests[0].values = vals;
    requests[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    cudf::groupby::groupby gb(cudf::table_view({keys}), cudf::null_policy::INCLUDE, cudf::sorted::YES);
    auto result = gb.aggregate(requests);
    auto kview  = result.first->view().column(0);
    expect_equal(host_valid(kview), std::vector<int>{1, 0, 1, 0, 1, 1}, "key validity");
    auto k = host_values<int32_t>(kview);
    expect_equal(std::vector<int32_t>{k[0], k[2], k[4], k[5]}, std::vector<int32_t>{1, 2, 3, 4}, "keys");
    expect_equal(host_values<int64_t>(result.second[0].results[0]->view()), std::vector<int64_t>{3, 7, 11, 7, 17, 4},
                 "sums");
  });
  run("structs_tests.cpp:124-148 structs_with_null_rows (STRUCT key with a STRING member)", [] {
    // members: int32 {1,2,3,1,2,2,1,3,3,2} and strings "11" / "22" / "33"; struct rows 0 and 3 null
    std::vector<int32_t> m0{1, 2, 3, 1, 2, 2, 1, 3, 3, 2};
    std::vector<std::string> m2{"11", "22", "33", "11", "22", "22", "11", "33", "33", "22"};
    std::string chars;
    std::vector<int32_t> offs{0};
    for (auto const& x : m2) {
      chars += x;
      offs.push_back(static_cast<int32_t>(chars.size()));
    }
    auto offsets = col(type_id::INT32, offs);
    cudf::column_view strings(cudf::data_type{type_id::STRING}, 10,
                              to_device(std::vector<char>(chars.begin(), chars.end())), nullptr, 0, 0, {offsets});
    std::vector<int> sv{0, 1, 1, 0, 1, 1, 1, 1, 1, 1};
    cudf::column_view key(cudf::data_type{type_id::STRUCT}, 10, nullptr, mask_of(sv), 2, 0,
                          {col(type_id::INT32, m0), strings});
    std::vector<cudf::groupby::aggregation_request> requests(1);
    requests[0].values = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9});
    requests[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    cudf::groupby::groupby gb(cudf::table_view({key}), cudf::null_policy::INCLUDE);
    auto result = gb.aggregate(requests);
    auto kv     = result.first->view().column(0);
    CHECK(kv.type().id() == type_id::STRUCT && kv.num_children() == 2, "a STRUCT key of two members");
    auto valid = host_valid(kv);
    auto sums  = host_values<int64_t>(result.second[0].results[0]->view());
    auto ints  = host_values<int32_t>(kv.child(0));
    auto ivld  = host_valid(kv.child(0));
    auto soffs = host_values<int32_t>(kv.child(1).child(0));
    std::vector<char> sch(static_cast<size_t>(soffs.back()));
    if (!sch.empty()) cudaMemcpy(sch.data(), kv.child(1).head(), sch.size(), cudaMemcpyDeviceToHost);
    CHECK(sums.size() == 4, "four groups");
    for (size_t g = 0; g < sums.size(); ++g) {
      if (!valid[g]) {
        CHECK(sums[g] == 3 && !ivld[g], "the null struct rows: sum 3, members null");
        continue;
      }
      const std::string s(sch.begin() + soffs[g], sch.begin() + soffs[g + 1]);
      const int64_t want = ints[g] == 1 ? 6 : ints[g] == 2 ? 19 : 17;
      CHECK(sums[g] == want && s == std::to_string(ints[g] * 11), "group %d", ints[g]);
    }
  });
  run("sum_tests.cpp:110-132 null_keys_and_values", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<double> v;
    run_single(col(type_id::INT32, K11, K11V),
               col(type_id::FLOAT64, std::vector<double>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4}, {0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0}),
               cudf::make_sum_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_equal(k, std::vector<int32_t>{1, 2, 3, 4}, "keys");
    expect_equal(vv, std::vector<int>{1, 1, 1, 0}, "validity");
    expect_near(v, {9, 14, 10, 0}, vv);
  });
  run("sum_tests.cpp:155-172 overflow_integer", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<int64_t> v;
    run_single(col(type_id::INT32, std::vector<int32_t>{0, 0}),
               col(type_id::INT32, std::vector<int32_t>{-2147483647 - 1, -2147483647 - 1}),
               cudf::make_sum_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_equal(v, std::vector<int64_t>{-4294967296LL}, "sum");
  });
  run("count_tests.cpp:116-145 null_keys_and_values (COUNT_ALL)", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<int32_t> v;
    run_single(col(type_id::INT32, K11, K11V),
               col(type_id::INT16, std::vector<int16_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4}, {0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0}),
               cudf::make_count_aggregation<cudf::groupby_aggregation>(cudf::null_policy::INCLUDE), k, kv, v, vv);
    expect_equal(v, std::vector<int32_t>{3, 4, 2, 1}, "counts");
  });
  run("max_tests.cpp:109-130 null_keys_and_values", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<int64_t> v;
    run_single(col(type_id::INT32, K11, K11V),
               col(type_id::INT64, std::vector<int64_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4}, {1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 0}),
               cudf::make_max_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_equal(vv, std::vector<int>{1, 1, 1, 0}, "validity");
    std::vector<int64_t> want{3, 5, 8};
    for (int i = 0; i < 3; ++i) CHECK(v[i] == want[i], "max[%d]", i);
  });
  run("mean_tests.cpp:48-64 basic", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<double> v;
    run_single(col(type_id::INT32, K10), col(type_id::INT8, std::vector<int8_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9}),
               cudf::make_mean_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_near(v, {3.0, 19.0 / 4, 17.0 / 3}, vv);
  });
  run("var_tests.cpp:126-148 ddof_non_default", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<double> v;
    run_single(col(type_id::INT32, K11, K11V),
               col(type_id::FLOAT32, std::vector<float>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 3}, {0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1}),
               cudf::make_variance_aggregation<cudf::groupby_aggregation>(2), k, kv, v, vv);
    expect_equal(vv, std::vector<int>{0, 1, 0, 0}, "validity");
    expect_near(v, {0, 98.0 / 3, 0, 0}, vv);
  });
  run("std_tests.cpp:35-53 basic", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<double> v;
    run_single(col(type_id::INT32, K10), col(type_id::INT64, std::vector<int64_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9}),
               cudf::make_std_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    expect_near(v, {3.0, std::sqrt(131.0 / 12), std::sqrt(31.0 / 3)}, vv);
  });
  run("keys_tests.cpp:94-120 include_null_keys", [] {
    std::vector<int64_t> k; std::vector<int> kv, vv; std::vector<int64_t> v;
    run_single(col(type_id::INT64, std::vector<int64_t>(K11.begin(), K11.end()), K11V),
               col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4}),
               cudf::make_sum_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv, cudf::null_policy::INCLUDE);
    expect_equal(kv, std::vector<int>{1, 1, 1, 1, 0}, "key validity");
    expect_equal(v, std::vector<int64_t>{9, 19, 10, 4, 7}, "sums");
  });
  run("keys_tests.cpp:338-365 dictionary keys", [] {
    // indices into the sorted dictionary {"aaa", "año", "₹1"}; the keys child is never read
    auto idx  = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 0, 1, 1, 0, 2, 2, 1});
    auto dkey = col(type_id::INT32, std::vector<int32_t>{0, 1, 2});
    cudf::column_view dict(cudf::data_type{type_id::DICTIONARY32}, 10, nullptr, nullptr, 0, 0, {idx, dkey});
    std::vector<cudf::groupby::aggregation_request> requests(1);
    requests[0].values = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9});
    requests[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    cudf::groupby::groupby gb(cudf::table_view({dict}));
    auto result = gb.aggregate(requests);
    auto kview  = result.first->view().column(0);
    CHECK(kview.type().id() == type_id::DICTIONARY32, "dictionary output keys");
    auto k = host_values<int32_t>(kview.child(0));
    auto v = host_values<int64_t>(result.second[0].results[0]->view());
    std::vector<int64_t> by_key(3);
    for (size_t i = 0; i < k.size(); ++i) by_key[k[i]] = v[i];
    expect_equal(by_key, std::vector<int64_t>{9, 19, 17}, "sums by dictionary index");
  });
  run("keys_tests.cpp:367-421 duplicate aggregations and columns", [] {
    auto keys = col(type_id::INT32, K10);
    auto vals = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4, 5, 6, 7, 8, 9});
    std::vector<cudf::groupby::aggregation_request> requests(2);
    requests[0].values = vals;
    requests[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    requests[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    requests[1].values = vals;
    requests[1].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
    cudf::groupby::groupby gb(cudf::table_view({keys}));
    auto result = gb.aggregate(requests);
    auto a = host_values<int64_t>(result.second[0].results[0]->view());
    auto b = host_values<int64_t>(result.second[0].results[1]->view());
    auto c = host_values<int64_t>(result.second[1].results[0]->view());
    expect_equal(a, b, "duplicate aggregation");
    expect_equal(a, c, "duplicate column");
  });
  run("keys_tests.cpp:227-243 mismatch_num_rows throws logic_error", [] {
    auto keys = col(type_id::INT32, std::vector<int32_t>{1, 2, 3});
    std::vector<cudf::groupby::aggregation_request> requests(1);
    requests[0].values = col(type_id::INT32, std::vector<int32_t>{0, 1, 2, 3, 4});
    requests[0].aggregations.push_back(cudf::make_count_aggregation<cudf::groupby_aggregation>());
    cudf::groupby::groupby gb(cudf::table_view({keys}));
    bool thrown = false;
    try {
      gb.aggregate(requests);
    } catch (cudf::logic_error const&) {
      thrown = true;
    }
    CHECK(thrown, "expected cudf::logic_error");
  });
  run("sum_tests.cpp:56-72 empty_cols", [] {
    std::vector<int32_t> k; std::vector<int> kv, vv; std::vector<int64_t> v;
    run_single(col(type_id::INT32, std::vector<int32_t>{}), col(type_id::INT32, std::vector<int32_t>{}),
               cudf::make_sum_aggregation<cudf::groupby_aggregation>(), k, kv, v, vv);
    CHECK(k.empty() && v.empty(), "empty result");
  });
  run("median / quantile / nunique / nth_element: median_tests.cpp:35 basic, quantile_tests.cpp:125, "
      "nunique_tests.cpp:31, nth_element_tests.cpp:94", [] {
    std::vector<int32_t> kk{1, 2, 3, 1, 2, 2, 1, 3, 3, 2};
    std::vector<int32_t> vv{0, 1, 2, 3, 4, 5, 6, 7, 8, 9};
    std::vector<int32_t> k; std::vector<int> kv, rv; std::vector<double> r;
    run_single(col(type_id::INT32, kk), col(type_id::INT32, vv),
               cudf::make_median_aggregation<cudf::groupby_aggregation>(), k, kv, r, rv);
    expect_near(r, {3., 4.5, 7.}, rv);
    std::vector<int32_t> nu; std::vector<int> nuv;
    run_single(col(type_id::INT32, kk), col(type_id::INT32, vv),
               cudf::make_nunique_aggregation<cudf::groupby_aggregation>(), k, kv, nu, nuv);
    expect_equal(nu, std::vector<int32_t>{3, 4, 3}, "nunique");
    std::vector<int32_t> nth; std::vector<int> nthv;
    run_single(col(type_id::INT32, kk), col(type_id::INT32, vv),
               cudf::make_nth_element_aggregation<cudf::groupby_aggregation>(-1), k, kv, nth, nthv);
    expect_equal(nth, std::vector<int32_t>{6, 9, 8}, "nth_element(-1)");
  });
  run("distinct_count_tests.cpp:279 TableWithSomeNull; distinct_tests.cpp:219 NoNullsTable", [] {
    auto c1 = col(type_id::INT32, std::vector<int32_t>{1, 2, 3, 4, 5, 6}, {1, 0, 1, 0, 1, 0});
    auto c2 = col(type_id::INT32, std::vector<int32_t>{1, 1, 1, 1, 1, 1});
    CHECK(cudf::distinct_count(cudf::table_view({c1, c2}), cudf::null_equality::EQUAL) == 4, "EQUAL");
    CHECK(cudf::distinct_count(cudf::table_view({c1, c2}), cudf::null_equality::UNEQUAL) == 6, "UNEQUAL");
    auto k1 = col(type_id::INT32, std::vector<int32_t>{20, 20, 20, 20, 19, 21, 9});
    auto k2 = col(type_id::INT32, std::vector<int32_t>{19, 19, 19, 20, 20, 9, 21});
    auto idx = cudf::distinct_indices(cudf::table_view({k1, k2}), cudf::duplicate_keep_option::KEEP_LAST);
    auto got = host_values<int32_t>(idx->view());
    std::sort(got.begin(), got.end());
    expect_equal(got, std::vector<int32_t>{2, 3, 4, 5, 6}, "KEEP_LAST rows");
  });
  run("distinct_join_tests.cpp:406 LeftJoinWithNulls (string keys as codes)", [] {
    auto b0 = col(type_id::INT32, std::vector<int32_t>{2, 2, 0, 4, 3});
    auto b1 = col(type_id::INT32, std::vector<int32_t>{1, 0, 1, 2, 1});
    auto p0 = col(type_id::INT32, std::vector<int32_t>{3, 1, 2, 0, 2});
    auto p1 = col(type_id::INT32, std::vector<int32_t>{1, 1, 0, 4, 0}, {1, 1, 0, 1, 1});
    cudf::distinct_hash_join join(cudf::table_view({b0, b1}), cudf::table_view({p0, p1}));
    auto left = host_values<int32_t>(join.left_join()->view());
    int32_t const none = std::numeric_limits<int32_t>::min();
    expect_equal(left, std::vector<int32_t>{4, none, none, none, 1}, "left join");
    auto [bi, pi] = join.inner_join();
    CHECK(bi->size() == 2 && pi->size() == 2, "two pairs");
  });
  run("join_tests.cpp:701-744 InnerJoinNoNulls (INT32 + STRING keys)", [] {
    auto strings = [](std::vector<std::string> const& v) {
      std::string chars;
      std::vector<int32_t> offs{0};
      for (auto const& x : v) {
        chars += x;
        offs.push_back(static_cast<int32_t>(chars.size()));
      }
      return cudf::column_view(cudf::data_type{type_id::STRING}, static_cast<cudf::size_type>(v.size()),
                               to_device(std::vector<char>(chars.begin(), chars.end())), nullptr, 0, 0,
                               {col(type_id::INT32, offs)});
    };
    auto l0 = col(type_id::INT32, std::vector<int32_t>{3, 1, 2, 0, 2});
    auto l1 = strings({"s1", "s1", "s0", "s4", "s0"});
    auto r0 = col(type_id::INT32, std::vector<int32_t>{2, 2, 0, 4, 3});
    auto r1 = strings({"s1", "s0", "s1", "s2", "s1"});
    auto [li, ri] = cudf::inner_join(cudf::table_view({l0, l1}), cudf::table_view({r0, r1}));
    auto a = host_values<int32_t>(li->view());
    auto b = host_values<int32_t>(ri->view());
    std::vector<std::pair<int32_t, int32_t>> pairs;
    for (size_t i = 0; i < a.size(); ++i) pairs.emplace_back(a[i], b[i]);
    std::sort(pairs.begin(), pairs.end());
    CHECK((pairs == std::vector<std::pair<int32_t, int32_t>>{{0, 4}, {2, 1}, {4, 1}}), "the matching pairs");
    auto semi = host_values<int32_t>(cudf::left_semi_join(cudf::table_view({l0, l1}),
                                                          cudf::table_view({r0, r1}))->view());
    std::sort(semi.begin(), semi.end());
    expect_equal(semi, std::vector<int32_t>{0, 2, 4}, "semi join");
  });
  for (auto p : g_buffers) cudaFree(p);
  std::printf("%d failure(s)\n", g_failures);
  return g_failures == 0 ? 0 : 1;
}
