// cudf/table/table.hpp -- an owning set of columns (cudf::table).
#pragma once

#include <memory>
#include <vector>

#include "../column/column.hpp"
#include "table_view.hpp"

namespace cudf {

class table {
 public:
  explicit table(std::vector<std::unique_ptr<column>>&& cols) : _columns(std::move(cols)) {}
  [[nodiscard]] size_type num_columns() const noexcept { return static_cast<size_type>(_columns.size()); }
  [[nodiscard]] size_type num_rows() const noexcept { return _columns.empty() ? 0 : _columns.front()->size(); }
  [[nodiscard]] table_view view() const
  {
    std::vector<column_view> v;
    for (auto const& c : _columns) v.push_back(c->view());
    return table_view(v);
  }
  column& get_column(size_type i) { return *_columns.at(i); }
  [[nodiscard]] column const& get_column(size_type i) const { return *_columns.at(i); }
  std::vector<std::unique_ptr<column>> release() { return std::move(_columns); }

 private:
  std::vector<std::unique_ptr<column>> _columns;
};

}  // namespace cudf
