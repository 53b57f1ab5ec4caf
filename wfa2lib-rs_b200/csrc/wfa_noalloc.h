// wfa_noalloc.h -- the fixed scratch array behind wfa_batch_align_device_noalloc.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wfa_b200.h"

namespace wfab {

constexpr size_t kNoAllocScratchBytes = WFA_NOALLOC_SCRATCH_BYTES;
constexpr int kNoAllocMaxDevices = 64;

// Device address of the array on `device`, which must be the current device.
// The first call for a device, and the first after its context was
// re-created (cudaDeviceReset), looks the address up (cudaGetSymbolAddress);
// later calls return the cached value.  Thread-safe.
cudaError_t noalloc_scratch(int device, int32_t** ptr);

}  // namespace wfab
