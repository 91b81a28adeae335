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
// device address is looked up with cudaGetSymbolAddress on every call, with
// the call's device current, and handed to the kernels as an ordinary
// pointer.  Looking it up per call (a few microseconds once the module is
// loaded) keeps it right after a device reset or a context re-created on the
// device, which unloads the module and would leave a cached address dangling.
//
// Under CUDA's lazy module loading (the default) neither this array nor the
// code of the kernels the call launches is on the device until first used.
// The set-up below therefore also loads every kernel the no-allocation path
// can launch, before the call does any work, so that all of the call's
// device memory is set aside at once -- by its first call on a device, which
// an empty input (zero rows) turns into a pure set-up call.  A caller that
// gives the GPU's memory to its own pool afterwards makes that first call
// beforehand, or runs with CUDA_MODULE_LOADING=EAGER.
#include <cuda_runtime.h>

#include "../../include/gbx.h"

namespace gbx {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GBX_NOALLOC_SCRATCH_BYTES];

cudaError_t load_noalloc_kernels();  // gbx_kernels.cu

// Device address of the scratch array on the current device, after loading
// the array and the kernels of the no-allocation path there.
cudaError_t noalloc_scratch(void** ptr, size_t* bytes)
{
  void* p       = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  if ((e = load_noalloc_kernels()) != cudaSuccess) return e;
  *ptr   = p;
  *bytes = sizeof(g_noalloc_scratch);
  return cudaSuccess;
}

}  // namespace gbx
