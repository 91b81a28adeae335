// cudf/stream_compaction.hpp -- distinct_count and distinct_indices with the
// reference's names and defaults (cpp/include/cudf/stream_compaction.hpp:
// 225-230, 311-317, 422-424), implemented over libgbx's C ABI (include/gbx.h).
#pragma once

#include <deque>
#include <memory>
#include <vector>

#include <rmm/cuda_stream_view.hpp>
#include <rmm/resource_ref.hpp>

#include "column/column.hpp"
#include "table/table_view.hpp"
#include "utilities/error.hpp"

namespace cudf {

enum class duplicate_keep_option { KEEP_ANY = 0, KEEP_FIRST, KEEP_LAST, KEEP_NONE };

namespace detail {
struct gbx_table_holder {
  std::vector<gbx_column_view> views;
  std::deque<std::vector<gbx_column_view>> store;  // dictionary keys, STRING offsets, STRUCT members
  gbx_table_view tv{};
  explicit gbx_table_holder(table_view const& t) : views(t.num_columns())
  {
    for (size_type i = 0; i < t.num_columns(); ++i) views[i] = t.column(i).to_gbx(store);
    tv.num_columns = t.num_columns();
    tv.columns     = views.data();
  }
};
}  // namespace detail

// The number of distinct rows (NaNs equal; under UNEQUAL every row holding a
// null is distinct).
inline size_type distinct_count(table_view const& input, null_equality nulls_equal = null_equality::EQUAL,
                                rmm::cuda_stream_view stream = rmm::cuda_stream_default)
{
  detail::gbx_table_holder h(input);
  int64_t out = 0;
  detail::throw_on_gbx_error(gbx_distinct_count(
    &h.tv, nulls_equal == null_equality::EQUAL ? GBX_NULLS_EQUAL : GBX_NULLS_UNEQUAL, stream.value(), nullptr, &out));
  return static_cast<size_type>(out);
}

// INT32 indices of the rows kept, one per distinct row, in no particular order.
inline std::unique_ptr<column> distinct_indices(
  table_view const& input, duplicate_keep_option keep = duplicate_keep_option::KEEP_ANY,
  null_equality nulls_equal = null_equality::EQUAL, nan_equality nans_equal = nan_equality::ALL_EQUAL,
  rmm::cuda_stream_view stream = rmm::cuda_stream_default,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  detail::gbx_table_holder h(input);
  gbx_column out{};
  detail::throw_on_gbx_error(gbx_distinct_indices(
    &h.tv, static_cast<int32_t>(keep), nulls_equal == null_equality::EQUAL ? GBX_NULLS_EQUAL : GBX_NULLS_UNEQUAL,
    nans_equal == nan_equality::ALL_EQUAL ? GBX_NANS_EQUAL : GBX_NANS_UNEQUAL, stream.value(), mr.allocator, &out));
  return std::make_unique<column>(out, mr.allocator, stream.value());
}

}  // namespace cudf
