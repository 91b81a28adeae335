// gbx_noalloc.cu -- fixed device scratch for gbx_groupby_aggregate_noalloc.
//
// Some callers cannot allocate device memory while they run a groupby: an
// engine that hands every byte of the GPU to its own pool at start-up and
// forbids other allocations, or a latency-critical thread where cudaMalloc /
// cudaFree would block or synchronise the device.  For them the hash table,
// the compaction map and the control words of one groupby live in this
// file-scope array instead of in allocated memory.  Every GPU that loads
// libgbx holds the array (GBX_NOALLOC_SCRATCH_BYTES) until the process exits.
//
// In host code `g_noalloc_scratch` only names a host-side stand-in for the
// symbol, never a device address: passing it to a kernel would fault, or,
// where the GPU can reach host memory, silently use the wrong memory.  The
// device address is obtained per device with cudaGetSymbolAddress, with that
// device current, and handed to the kernels as an ordinary pointer.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gbx.h"

namespace gbx {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GBX_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};
}  // namespace

// Device address of the scratch array on `device`, which must be the current
// device.  The lookup runs once per device (the first no-alloc call on it).
cudaError_t noalloc_scratch(int device, void** ptr, size_t* bytes)
{
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[device] == nullptr) {
    void* p       = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = p;
  }
  *ptr   = g_addr[device];
  *bytes = sizeof(g_noalloc_scratch);
  return cudaSuccess;
}

}  // namespace gbx
