// cudf/join.hpp -- the hash joins inner_join / left_join / full_join /
// left_semi_join / left_anti_join (cpp/include/cudf/join.hpp:107-260) and
// distinct_hash_join with the reference's constructor and inner_join /
// left_join (:475-533), implemented over libgbx's C ABI (include/gbx.h).  The
// index vectors come back as INT32 columns; a row without a match on the
// other side is INT32_MIN (JoinNoneValue).
#pragma once

#include <memory>
#include <utility>

#include <rmm/cuda_stream_view.hpp>
#include <rmm/resource_ref.hpp>

#include "column/column.hpp"
#include "stream_compaction.hpp"
#include "table/table_view.hpp"
#include "utilities/error.hpp"

namespace cudf {

enum class nullable_join : bool { YES, NO };

namespace detail {
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> hash_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls, gbx_join_kind kind,
  rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr)
{
  gbx_table_holder hl(left_keys), hr(right_keys);
  gbx_column l{}, r{};
  throw_on_gbx_error(gbx_hash_join(&hl.tv, &hr.tv,
                                   compare_nulls == null_equality::EQUAL ? GBX_NULLS_EQUAL : GBX_NULLS_UNEQUAL,
                                   kind, stream.value(), mr.allocator, &l, &r));
  return {std::make_unique<column>(l, mr.allocator, stream.value()),
          std::make_unique<column>(r, mr.allocator, stream.value())};
}
}  // namespace detail

// join.hpp:107-112: (left rows, right rows) of every matching pair
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> inner_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls = null_equality::EQUAL,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  return detail::hash_join(left_keys, right_keys, compare_nulls, GBX_JOIN_INNER, rmm::cuda_stream_default, mr);
}

// join.hpp:147-152: every left row with each matching right row, or JoinNoneValue
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> left_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls = null_equality::EQUAL,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  return detail::hash_join(left_keys, right_keys, compare_nulls, GBX_JOIN_LEFT, rmm::cuda_stream_default, mr);
}

// join.hpp:186-191: the left join's pairs, then (JoinNoneValue, right row) for unmatched right rows
inline std::pair<std::unique_ptr<column>, std::unique_ptr<column>> full_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls = null_equality::EQUAL,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  return detail::hash_join(left_keys, right_keys, compare_nulls, GBX_JOIN_FULL, rmm::cuda_stream_default, mr);
}

// join.hpp:215-219: the left rows that have a match
inline std::unique_ptr<column> left_semi_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls = null_equality::EQUAL,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  return detail::hash_join(left_keys, right_keys, compare_nulls, GBX_JOIN_LEFT_SEMI, rmm::cuda_stream_default, mr)
    .first;
}

// join.hpp:246-250: the left rows that have no match
inline std::unique_ptr<column> left_anti_join(
  table_view const& left_keys, table_view const& right_keys, null_equality compare_nulls = null_equality::EQUAL,
  rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource())
{
  return detail::hash_join(left_keys, right_keys, compare_nulls, GBX_JOIN_LEFT_ANTI, rmm::cuda_stream_default, mr)
    .first;
}

class distinct_hash_join {
 public:
  distinct_hash_join(table_view const& build, table_view const& probe, nullable_join = nullable_join::YES,
                     null_equality compare_nulls = null_equality::EQUAL,
                     rmm::cuda_stream_view stream = rmm::cuda_stream_default)
    : _build(build), _probe(probe), _compare(compare_nulls), _stream(stream)
  {
  }
  distinct_hash_join(distinct_hash_join const&)            = delete;
  distinct_hash_join& operator=(distinct_hash_join const&) = delete;

  // [build_indices, probe_indices] of the matching row pairs
  [[nodiscard]] std::pair<std::unique_ptr<column>, std::unique_ptr<column>> inner_join(
    rmm::cuda_stream_view stream = rmm::cuda_stream_default,
    rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource()) const
  {
    gbx_column b{}, p{};
    run(0, stream, mr, b, p);
    return {std::make_unique<column>(b, mr.allocator, stream.value()),
            std::make_unique<column>(p, mr.allocator, stream.value())};
  }

  // the build row of every probe row (INT32_MIN: none)
  [[nodiscard]] std::unique_ptr<column> left_join(
    rmm::cuda_stream_view stream = rmm::cuda_stream_default,
    rmm::device_async_resource_ref mr = rmm::mr::get_current_device_resource()) const
  {
    gbx_column b{}, p{};
    run(1, stream, mr, b, p);
    column discard(p, mr.allocator, stream.value());
    return std::make_unique<column>(b, mr.allocator, stream.value());
  }

 private:
  void run(int kind, rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr, gbx_column& b,
           gbx_column& p) const
  {
    detail::gbx_table_holder hb(_build), hp(_probe);
    detail::throw_on_gbx_error(gbx_distinct_join(
      &hb.tv, &hp.tv, _compare == null_equality::EQUAL ? GBX_NULLS_EQUAL : GBX_NULLS_UNEQUAL, kind, stream.value(),
      mr.allocator, &b, &p));
  }
  table_view _build, _probe;
  null_equality _compare;
  rmm::cuda_stream_view _stream;
};

}  // namespace cudf
