// cudf/join.hpp -- distinct_hash_join with the reference's constructor and
// inner_join / left_join (cpp/include/cudf/join.hpp:475-533), implemented over
// libgbx's C ABI (include/gbx.h).  The index vectors come back as INT32
// columns; a left join marks probe rows without a match with INT32_MIN
// (JoinNoneValue).
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
