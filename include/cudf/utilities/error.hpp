// cudf/utilities/error.hpp -- the exception types of the reference
// (cpp/include/cudf/utilities/error.hpp:64, 92) and the mapping from libgbx
// status codes to them.
#pragma once

#include <stdexcept>
#include <string>

#include "../../gbx.h"

namespace cudf {

struct logic_error : public std::logic_error {
  using std::logic_error::logic_error;
};

struct cuda_error : public std::runtime_error {
  using std::runtime_error::runtime_error;
};

namespace detail {
// Throws the reference's exception type for a non-zero gbx_status.
inline void throw_on_gbx_error(int status)
{
  if (status == GBX_OK) return;
  std::string msg = gbx_last_error();
  if (status == GBX_ERR_CUDA || status == GBX_ERR_DEVICE) throw cuda_error("CUDA error: " + msg);
  if (status == GBX_ERR_ALLOC) throw std::bad_alloc();
  throw logic_error("cuDF failure: " + msg);
}
}  // namespace detail

}  // namespace cudf
