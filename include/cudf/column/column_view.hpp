// cudf/column/column_view.hpp -- a non-owning column description with the
// reference's accessors (cpp/include/cudf/column/column_view.hpp).  A
// DICTIONARY32 view has two children: 0 = indices, 1 = keys; a STRING view
// holds its characters in the data buffer and child 0 = offsets; a STRUCT
// view's children are its members.
#pragma once

#include <deque>
#include <vector>

#include "../types.hpp"

namespace cudf {

class column_view {
 public:
  column_view() = default;
  column_view(data_type type, size_type size, void const* data, bitmask_type const* null_mask = nullptr,
              size_type null_count = 0, size_type offset = 0, std::vector<column_view> const& children = {})
    : _type(type), _size(size), _data(data), _null_mask(null_mask), _null_count(null_count), _offset(offset),
      _children(children)
  {
  }
  [[nodiscard]] data_type type() const noexcept { return _type; }
  [[nodiscard]] size_type size() const noexcept { return _size; }
  [[nodiscard]] bool is_empty() const noexcept { return _size == 0; }
  [[nodiscard]] size_type offset() const noexcept { return _offset; }
  [[nodiscard]] bitmask_type const* null_mask() const noexcept { return _null_mask; }
  [[nodiscard]] bool nullable() const noexcept { return _null_mask != nullptr; }
  [[nodiscard]] size_type null_count() const noexcept { return _null_count; }
  [[nodiscard]] bool has_nulls() const noexcept { return null_count() > 0; }
  [[nodiscard]] void const* head() const noexcept { return _data; }
  template <typename T>
  [[nodiscard]] T const* data() const noexcept
  {
    return static_cast<T const*>(_data) + _offset;
  }
  [[nodiscard]] size_type num_children() const noexcept { return static_cast<size_type>(_children.size()); }
  [[nodiscard]] column_view child(size_type i) const { return _children.at(i); }

  // The C-ABI descriptor of this view; `keys_storage` receives the dictionary
  // keys' descriptor and must outlive the returned value.
  gbx_column_view to_gbx(gbx_column_view* keys_storage) const
  {
    gbx_column_view v{};
    v.type_id    = static_cast<int32_t>(_type.id());
    v.scale      = _type.scale();
    v.size       = _size;
    v.offset     = _offset;
    v.data       = _data;
    v.null_mask  = _null_mask;
    v.null_count = _null_mask ? _null_count : 0;
    if (_type.id() == type_id::DICTIONARY32 && _children.size() == 2) {
      column_view const& idx = _children[0];
      v.data                 = idx.head();
      v.offset               = _offset + idx.offset();
      v.index_type_id        = static_cast<int32_t>(idx.type().id());
      *keys_storage          = _children[1].to_gbx(nullptr);
      v.dict_keys            = keys_storage;
    }
    return v;
  }

  // The C-ABI descriptor of this view for any supported type: the
  // descriptors it points at (dictionary keys, STRING offsets, STRUCT
  // members) are kept in `store`, which must outlive the returned value.
  gbx_column_view to_gbx(std::deque<std::vector<gbx_column_view>>& store) const
  {
    if (_type.id() == type_id::DICTIONARY32) {
      store.emplace_back(1);
      return to_gbx(store.back().data());
    }
    gbx_column_view v{};
    v.type_id    = static_cast<int32_t>(_type.id());
    v.scale      = _type.scale();
    v.size       = _size;
    v.offset     = _offset;
    v.data       = _data;
    v.null_mask  = _null_mask;
    v.null_count = _null_mask ? _null_count : 0;
    if (_type.id() == type_id::STRING && !_children.empty()) {
      gbx_column_view offsets = _children[0].to_gbx(store);
      store.emplace_back(1, offsets);
      v.dict_keys = store.back().data();
    } else if (_type.id() == type_id::STRUCT) {
      std::vector<gbx_column_view> members;
      for (auto const& c : _children) members.push_back(c.to_gbx(store));
      store.push_back(std::move(members));
      v.data         = nullptr;
      v.num_children = static_cast<int32_t>(store.back().size());
      v.dict_keys    = store.back().data();
    }
    return v;
  }

  // A view of a C-ABI descriptor (STRING offsets and STRUCT members as
  // children), borrowing its buffers.
  static column_view from_gbx(gbx_column_view const& v)
  {
    data_type t{static_cast<type_id>(v.type_id), v.scale};
    auto const size = static_cast<size_type>(v.size);
    auto const nc   = static_cast<size_type>(v.null_count < 0 ? 0 : v.null_count);
    auto const off  = static_cast<size_type>(v.offset);
    std::vector<column_view> kids;
    if (v.type_id == GBX_TYPE_STRING && v.dict_keys != nullptr) {
      kids.push_back(from_gbx(*v.dict_keys));
    } else if (v.type_id == GBX_TYPE_STRUCT) {
      for (int32_t m = 0; m < v.num_children; ++m) kids.push_back(from_gbx(v.dict_keys[m]));
    }
    return column_view(t, size, v.type_id == GBX_TYPE_STRUCT ? nullptr : v.data,
                       static_cast<bitmask_type const*>(v.null_mask), nc, off, kids);
  }

 private:
  data_type _type{type_id::EMPTY};
  size_type _size{};
  void const* _data{};
  bitmask_type const* _null_mask{};
  size_type _null_count{};
  size_type _offset{};
  std::vector<column_view> _children{};
};

}  // namespace cudf
