// cudf/utilities/span.hpp -- host_span (cpp/include/cudf/utilities/span.hpp).
#pragma once

#include <cstddef>
#include <vector>

namespace cudf {

template <typename T>
class host_span {
 public:
  constexpr host_span() noexcept = default;
  constexpr host_span(T* data, std::size_t size) noexcept : _data(data), _size(size) {}
  template <typename C, typename = decltype(std::declval<C&>().data())>
  constexpr host_span(C& c) noexcept : _data(c.data()), _size(c.size())
  {
  }
  template <typename C, typename = decltype(std::declval<C const&>().data())>
  constexpr host_span(C const& c) noexcept : _data(c.data()), _size(c.size())
  {
  }
  [[nodiscard]] constexpr T* data() const noexcept { return _data; }
  [[nodiscard]] constexpr std::size_t size() const noexcept { return _size; }
  [[nodiscard]] constexpr bool empty() const noexcept { return _size == 0; }
  constexpr T& operator[](std::size_t i) const { return _data[i]; }
  constexpr T* begin() const noexcept { return _data; }
  constexpr T* end() const noexcept { return _data + _size; }

 private:
  T* _data{nullptr};
  std::size_t _size{0};
};

}  // namespace cudf
