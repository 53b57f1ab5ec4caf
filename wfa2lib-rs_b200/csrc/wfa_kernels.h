// wfa_kernels.h -- kernel launchers used by the host side.
#pragma once
#include <cuda_runtime.h>

#include "wfa_common.h"

namespace wfab {

constexpr int kWarpsPerBlock = 4;

// Size in bytes of one warp's wavefront-descriptor ring (shared memory).
inline size_t ring_desc_bytes(int scope, int nc) { return (size_t)scope * nc * 32; }

cudaError_t launch_unialign(const AlignParams& P, int metric_class, int blocks, size_t smem,
                            cudaStream_t st);
int occupancy_blocks_per_sm(int metric_class, bool packed, size_t smem);

}  // namespace wfab
