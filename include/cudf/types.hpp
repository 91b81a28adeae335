// cudf/types.hpp -- the subset of libcudf's core types the groupby facade
// uses, with the reference's names and values (cpp/include/cudf/types.hpp:95-235).
#pragma once

#include <cstdint>

#include "../gbx.h"

namespace cudf {

using size_type    = int32_t;   // types.hpp:95
using bitmask_type = uint32_t;  // types.hpp:96

enum class null_policy : bool { EXCLUDE, INCLUDE };  // types.hpp:126
enum class interpolation : int32_t { LINEAR, LOWER, HIGHER, MIDPOINT, NEAREST };  // types.hpp:192-198
enum class sorted : bool { NO, YES };                // types.hpp:167
enum class order : bool { ASCENDING, DESCENDING };
enum class null_order : bool { AFTER, BEFORE };
enum class null_equality : bool { EQUAL, UNEQUAL };  // types.hpp:151-154
enum class nan_equality { ALL_EQUAL, UNEQUAL };      // types.hpp:143-146

enum class type_id : int32_t {
  EMPTY = GBX_TYPE_EMPTY,
  INT8,
  INT16,
  INT32,
  INT64,
  UINT8,
  UINT16,
  UINT32,
  UINT64,
  FLOAT32,
  FLOAT64,
  BOOL8,
  TIMESTAMP_DAYS,
  TIMESTAMP_SECONDS,
  TIMESTAMP_MILLISECONDS,
  TIMESTAMP_MICROSECONDS,
  TIMESTAMP_NANOSECONDS,
  DURATION_DAYS,
  DURATION_SECONDS,
  DURATION_MILLISECONDS,
  DURATION_MICROSECONDS,
  DURATION_NANOSECONDS,
  DICTIONARY32,
  STRING,
  LIST,
  DECIMAL32,
  DECIMAL64,
  DECIMAL128,
  STRUCT,
  NUM_TYPE_IDS
};

class data_type {
 public:
  data_type() = default;
  explicit constexpr data_type(type_id id) : _id{id} {}
  constexpr data_type(type_id id, int32_t scale) : _id{id}, _fixed_point_scale{scale} {}
  [[nodiscard]] constexpr type_id id() const noexcept { return _id; }
  [[nodiscard]] constexpr int32_t scale() const noexcept { return _fixed_point_scale; }
  constexpr bool operator==(data_type const& o) const { return _id == o._id && _fixed_point_scale == o._fixed_point_scale; }
  constexpr bool operator!=(data_type const& o) const { return !(*this == o); }

 private:
  type_id _id{type_id::EMPTY};
  int32_t _fixed_point_scale{};
};

inline std::size_t size_of(data_type t)
{
  switch (t.id()) {
    case type_id::INT8:
    case type_id::UINT8:
    case type_id::BOOL8: return 1;
    case type_id::INT16:
    case type_id::UINT16: return 2;
    case type_id::INT32:
    case type_id::UINT32:
    case type_id::FLOAT32:
    case type_id::TIMESTAMP_DAYS:
    case type_id::DURATION_DAYS:
    case type_id::DECIMAL32:
    case type_id::DICTIONARY32: return 4;
    case type_id::EMPTY:
    case type_id::STRING:
    case type_id::LIST:
    case type_id::STRUCT:
    case type_id::NUM_TYPE_IDS: return 0;
    case type_id::DECIMAL128: return 16;
    default: return 8;
  }
}

}  // namespace cudf
