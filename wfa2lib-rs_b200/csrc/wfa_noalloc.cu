// wfa_noalloc.cu -- the scratch of the no-allocation batch entry point: one
// file-scope device array of WFA_NOALLOC_SCRATCH_BYTES.  It belongs to this
// file's module, so a device holds it from the first use of the entry point
// there until the process exits; the other entry points never touch it.
#include <mutex>

#include "wfa_noalloc.h"

namespace wfab {

static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocScratchBytes / 4];

static std::mutex g_noalloc_mu;
static int32_t* g_noalloc_addr[kNoAllocMaxDevices];

// In host code `g_noalloc_scratch` names a host-side stand-in, not device
// memory, so the kernels get the device address looked up here, once per
// device, with that device current.
cudaError_t noalloc_scratch(int device, int32_t** ptr) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[device] = static_cast<int32_t*>(p);
  }
  *ptr = g_noalloc_addr[device];
  return cudaSuccess;
}

}  // namespace wfab
