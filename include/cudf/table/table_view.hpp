// cudf/table/table_view.hpp -- an ordered set of column_views (cudf::table_view).
#pragma once

#include <initializer_list>
#include <vector>

#include "../column/column_view.hpp"

namespace cudf {

class table_view {
 public:
  table_view() = default;
  table_view(std::vector<column_view> const& cols) : _columns(cols) {}
  table_view(std::initializer_list<column_view> cols) : _columns(cols) {}
  [[nodiscard]] size_type num_columns() const noexcept { return static_cast<size_type>(_columns.size()); }
  [[nodiscard]] size_type num_rows() const noexcept { return _columns.empty() ? 0 : _columns.front().size(); }
  [[nodiscard]] column_view const& column(size_type i) const { return _columns.at(i); }
  [[nodiscard]] auto begin() const noexcept { return _columns.begin(); }
  [[nodiscard]] auto end() const noexcept { return _columns.end(); }

 private:
  std::vector<column_view> _columns;
};

}  // namespace cudf
