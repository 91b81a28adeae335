// gbx_scan.hpp -- device-wide exclusive scans and occupied-slot compaction
// (gbx_scan.cu), libgbx's own kernels in place of library scans and selects.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace gbx {

struct TableRef;

// out[i] = in[0] + ... + in[i-1] for i < n (out may alias in).  Called with
// temp == nullptr it only stores the scratch size it needs in *temp_bytes.
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, void* temp, size_t* temp_bytes,
                               cudaStream_t st);
cudaError_t scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, void* temp, size_t* temp_bytes,
                               cudaStream_t st);

// Kernels one scan of n values launches.
int scan_launches(int64_t n);

}  // namespace gbx
