// cudf/groupby.hpp -- cudf::groupby::groupby with the reference's signatures
// (cpp/include/cudf/groupby.hpp:61-199), implemented over libgbx's C ABI
// (include/gbx.h).  Link with -lgbx.
#pragma once

#include <cuda_runtime_api.h>

#include <memory>
#include <utility>
#include <vector>

#include <rmm/cuda_stream_view.hpp>
#include <rmm/resource_ref.hpp>

#include "aggregation.hpp"
#include "column/column.hpp"
#include "table/table.hpp"
#include "table/table_view.hpp"
#include "utilities/error.hpp"
#include "utilities/span.hpp"

namespace cudf {
namespace groupby {

// groupby.hpp:61-64
struct aggregation_request {
  column_view values;
  std::vector<std::unique_ptr<groupby_aggregation>> aggregations;
};

// groupby.hpp:88-91
struct aggregation_result {
  std::vector<std::unique_ptr<column>> results{};
};

class groupby {
 public:
  groupby()                          = delete;
  groupby(groupby const&)            = delete;
  groupby(groupby&&)                 = delete;
  groupby& operator=(groupby const&) = delete;
  groupby& operator=(groupby&&)      = delete;

  // groupby.hpp:128-132.  Borrows `keys`: the caller keeps the data alive.
  explicit groupby(table_view const& keys,
                   null_policy null_handling                      = null_policy::EXCLUDE,
                   sorted keys_are_sorted                         = sorted::NO,
                   std::vector<order> const& column_order         = {},
                   std::vector<null_order> const& null_precedence = {})
    : _keys(keys)
  {
    (void)column_order;
    (void)null_precedence;
    _kviews.resize(keys.num_columns());
    for (size_type i = 0; i < keys.num_columns(); ++i) _kviews[i] = keys.column(i).to_gbx(_kstore);
    gbx_table_view tv{};
    tv.num_columns = keys.num_columns();
    tv.columns     = _kviews.data();
    detail::throw_on_gbx_error(gbx_groupby_create(&tv, null_handling == null_policy::INCLUDE ? 1 : 0,
                                                  keys_are_sorted == sorted::YES ? 1 : 0, &_gb));
  }
  ~groupby() { gbx_groupby_destroy(_gb); }

  // groupby.hpp:187-190
  std::pair<std::unique_ptr<table>, std::vector<aggregation_result>> aggregate(
    host_span<aggregation_request const> requests,
    rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
  {
    return aggregate(requests, rmm::cuda_stream_default, mr);
  }

  // groupby.hpp:196-199
  std::pair<std::unique_ptr<table>, std::vector<aggregation_result>> aggregate(
    host_span<aggregation_request const> requests,
    rmm::cuda_stream_view stream,
    rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
  {
    std::vector<gbx_request> reqs(requests.size());
    std::vector<gbx_column_view> dict(requests.size());
    std::vector<std::vector<gbx_aggregation>> aggs(requests.size());
    for (std::size_t i = 0; i < requests.size(); ++i) {
      reqs[i].values = requests[i].values.to_gbx(&dict[i]);
      for (auto const& a : requests[i].aggregations) {
        gbx_aggregation g{};
        g.kind          = static_cast<int32_t>(a->kind);
        g.ddof          = a->ddof;
        g.null_policy   = a->null_handling == null_policy::INCLUDE ? GBX_NULL_INCLUDE : GBX_NULL_EXCLUDE;
        g.interpolation = static_cast<int32_t>(a->interp);
        g.num_quantiles = static_cast<int32_t>(a->quantiles.size());
        g.quantiles     = a->quantiles.data();
        aggs[i].push_back(g);
      }
      reqs[i].num_aggregations = static_cast<int32_t>(aggs[i].size());
      reqs[i].aggregations     = aggs[i].data();
    }
    gbx_result* res = nullptr;
    detail::throw_on_gbx_error(gbx_groupby_aggregate(_gb, reqs.data(), static_cast<int32_t>(reqs.size()),
                                                     stream.value(), mr.allocator, &res));
    // move every buffer into its own owning column, then free the shell
    // (kept while a STRING / STRUCT key column points into it)
    std::shared_ptr<void> shell(res, [](void* r) { gbx_result_release(static_cast<gbx_result*>(r)); });
    std::vector<std::unique_ptr<column>> key_cols;
    for (int c = 0; c < res->num_key_columns; ++c) {
      column_view dk = _keys.column(c).type().id() == type_id::DICTIONARY32 ? _keys.column(c).child(1) : column_view{};
      const auto kt  = _keys.column(c).type().id();
      key_cols.push_back(std::make_unique<column>(res->keys[c], mr.allocator, stream.value(), dk,
                                                  kt == type_id::STRING || kt == type_id::STRUCT ? shell : nullptr));
      res->keys[c].data      = nullptr;
      res->keys[c].null_mask = nullptr;
    }
    std::vector<aggregation_result> out(res->num_requests);
    for (int q = 0; q < res->num_requests; ++q) {
      for (int k = 0; k < res->requests[q].num_results; ++k) {
        gbx_column& gc = res->requests[q].results[k];
        out[q].results.push_back(std::make_unique<column>(gc, mr.allocator, stream.value(), column_view{},
                                                          gc.view.type_id == GBX_TYPE_STRING ? shell : nullptr));
        gc.data      = nullptr;
        gc.null_mask = nullptr;
      }
    }
    return {std::make_unique<table>(std::move(key_cols)), std::move(out)};
  }

 private:
  table_view _keys;
  std::vector<gbx_column_view> _kviews;
  std::deque<std::vector<gbx_column_view>> _kstore;
  gbx_groupby* _gb{nullptr};
};

}  // namespace groupby
}  // namespace cudf
