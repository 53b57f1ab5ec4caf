// wfa_kernels.h -- kernel launchers used by the host side.
#pragma once
#include <cuda_runtime.h>

#include "wfa_common.h"

namespace wfab {

constexpr int kWarpsPerBlock = 4;
constexpr int kMinBlocksPerSM = 6;  // register budget: 65536 / (6 * 128) = 85 per thread
constexpr int kDescBytes = 32;      // sizeof(WfD)

// Per-block dynamic shared memory: descriptor rings, staged sequences and
// (optionally) ring cells, each as kWarpsPerBlock per-warp slices.
struct SmemLayout {
  size_t desc_bytes, seq_bytes, ring_bytes;  // per warp
  size_t desc_off, seq_off, ring_off, total;  // per block
};
#if defined(__CUDACC__)
__host__ __device__
#endif
inline SmemLayout smem_layout(int scope, int nc, int ring_wmax, int seq_words) {
  SmemLayout L;
  L.desc_bytes = (size_t)scope * nc * kDescBytes;
  L.seq_bytes = (size_t)2 * seq_words * 4;
  L.ring_bytes = (size_t)scope * nc * ring_wmax * 4;
  L.desc_off = 0;
  L.seq_off = L.desc_off + kWarpsPerBlock * L.desc_bytes;
  L.ring_off = L.seq_off + kWarpsPerBlock * L.seq_bytes;
  L.total = L.ring_off + kWarpsPerBlock * L.ring_bytes;
  return L;
}

bool needs_general(const AlignParams& P);
cudaError_t launch_unialign(const AlignParams& P, int metric_class, int blocks, size_t smem,
                            cudaStream_t st);
int occupancy_blocks_per_sm(const AlignParams& P, int metric_class, size_t smem);

}  // namespace wfab
