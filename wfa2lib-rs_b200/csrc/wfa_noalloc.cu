// wfa_noalloc.cu -- the scratch of the no-allocation batch entry point: one
// file-scope device array of WFA_NOALLOC_SCRATCH_BYTES.  It belongs to this
// file's module, so a device holds it from the first use of the entry point
// there until the process exits; the other entry points never touch it.
#include <cuda.h>
#include <mutex>

#include "wfa_noalloc.h"

namespace wfab {

static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocScratchBytes / 4];

// The array's device address, looked up per device and remembered with the
// identity of the context it was looked up in.  A program that resets a
// device (cudaDeviceReset) gets a new primary context, in which the module
// is loaded again and the array can sit elsewhere: the next call sees a new
// context id and looks the address up again instead of using a stale one.
struct NoAllocSlot {
  unsigned long long ctx_id;
  int32_t* addr;
};
static std::mutex g_noalloc_mu;
static NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the current context (cuCtxGetId, reached through the runtime's
// driver entry points so the library needs no link against libcuda).
static cudaError_t current_ctx_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
    if (e != cudaSuccess) return e;
    e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
    if (e != cudaSuccess) return e;
    if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
      return cudaErrorNotSupported;
    get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
    get_id = reinterpret_cast<CtxGetIdFn>(f1);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
  if (get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  return cudaSuccess;
}

// In host code `g_noalloc_scratch` names a host-side stand-in, not device
// memory, so the kernels get the device address looked up here, with the
// device current: once per device and context.
cudaError_t noalloc_scratch(int device, int32_t** ptr) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  // The caller has made the device current (cudaSetDevice, which also makes
  // its primary context current).
  unsigned long long id = 0;
  cudaError_t e = current_ctx_id(&id);
  if (e != cudaSuccess) return e;
  NoAllocSlot& s = g_noalloc_slot[device];
  if (!s.addr || s.ctx_id != id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    s.addr = static_cast<int32_t*>(p);
    s.ctx_id = id;
  }
  *ptr = s.addr;
  return cudaSuccess;
}

}  // namespace wfab
