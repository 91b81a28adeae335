// cudf/column/column.hpp -- an owning device column (cudf::column) holding
// one result buffer (and mask) released through the allocator it came from.
#pragma once

#include <cuda_runtime_api.h>

#include <memory>

#include "column_view.hpp"

namespace cudf {

class column {
 public:
  column()              = default;
  column(column const&) = delete;
  column& operator=(column const&) = delete;

  // Adopts a result column produced by libgbx.  `keep` holds what the
  // column's children point into (a STRING key's offsets, a STRUCT key's
  // members: buffers the libgbx result owns).
  column(gbx_column const& c, gbx_allocator const* mr, cudaStream_t stream, column_view dict_keys = {},
         std::shared_ptr<void> keep = {})
    : _c(c), _has_mr(mr != nullptr), _stream(stream), _dict_keys(dict_keys), _keep(std::move(keep))
  {
    if (mr) _mr = *mr;
  }
  ~column()
  {
    release_buffer(_c.data, _c.data_bytes);
    release_buffer(_c.null_mask, _c.mask_bytes);
  }

  [[nodiscard]] data_type type() const noexcept { return data_type{static_cast<type_id>(_c.view.type_id), _c.view.scale}; }
  [[nodiscard]] size_type size() const noexcept { return static_cast<size_type>(_c.view.size); }
  [[nodiscard]] size_type null_count() const noexcept { return static_cast<size_type>(_c.view.null_count < 0 ? 0 : _c.view.null_count); }
  [[nodiscard]] bool nullable() const noexcept { return _c.null_mask != nullptr; }
  [[nodiscard]] bool has_nulls() const noexcept { return null_count() > 0; }

  [[nodiscard]] column_view view() const
  {
    auto t = type();
    if (t.id() == type_id::DICTIONARY32) {
      data_type it{static_cast<type_id>(_c.view.index_type_id ? _c.view.index_type_id : GBX_TYPE_INT32)};
      column_view indices(it, size(), _c.data);
      return column_view(t, size(), nullptr, _c.null_mask, null_count(), 0, {indices, _dict_keys});
    }
    if (t.id() == type_id::STRING || t.id() == type_id::STRUCT) {
      gbx_column_view v = _c.view;
      v.data            = _c.data;
      v.null_mask       = _c.null_mask;
      return column_view::from_gbx(v);
    }
    return column_view(t, size(), _c.data, _c.null_mask, null_count());
  }
  operator column_view() const { return view(); }

 private:
  void release_buffer(void* p, size_t bytes)
  {
    if (!p) return;
    bytes = (bytes == 0 ? 8 : bytes);
    bytes = (bytes + 255) & ~size_t(255);
    if (_has_mr) _mr.deallocate(_mr.ctx, p, bytes, _stream);
    else cudaFreeAsync(p, _stream);
  }
  gbx_column _c{};
  gbx_allocator _mr{};
  bool _has_mr{false};
  cudaStream_t _stream{nullptr};
  column_view _dict_keys{};
  std::shared_ptr<void> _keep{};
};

}  // namespace cudf
