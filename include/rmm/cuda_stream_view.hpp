// rmm/cuda_stream_view.hpp -- the stream handle the groupby API takes
// (rmm::cuda_stream_view), reduced to what the facade needs.
#pragma once

#include <cuda_runtime_api.h>

namespace rmm {

class cuda_stream_view {
 public:
  constexpr cuda_stream_view() = default;
  constexpr cuda_stream_view(cudaStream_t s) noexcept : _s(s) {}
  [[nodiscard]] constexpr cudaStream_t value() const noexcept { return _s; }
  constexpr operator cudaStream_t() const noexcept { return _s; }
  void synchronize() const { cudaStreamSynchronize(_s); }

 private:
  cudaStream_t _s{nullptr};
};

inline cuda_stream_view cuda_stream_default{};

}  // namespace rmm
