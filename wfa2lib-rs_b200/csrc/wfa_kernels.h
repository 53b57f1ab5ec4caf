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

// BiWFA per-warp scratch slice (int32 word offsets).  seq_len_sum is the
// longest n + m of the launch (sizes the reversed sequences and the base CIGAR).
// The forward and reverse rings are wmax cells wide; the base-case ring only
// wmax_base: a base case ends by score 500 (plus one scope), and a wavefront
// at score s spans at most 2s + 1 diagonals.
struct BiLayout {
  int64_t ring_f, ring_r, ring_b, hist, harena, rev, cig, words;
};
#if defined(__CUDACC__)
__host__ __device__
#endif
inline BiLayout bi_layout(int scope, int nc, int wmax, int wmax_base, int hist_scores,
                          int64_t hist_words, int seq_len_sum) {
  BiLayout L;
  const int64_t ring = ((int64_t)scope * nc * wmax + 3) & ~(int64_t)3;
  const int64_t ring_b = ((int64_t)scope * nc * wmax_base + 3) & ~(int64_t)3;
  L.ring_f = 0;
  L.ring_r = L.ring_f + ring;
  L.ring_b = L.ring_r + ring;
  L.hist = L.ring_b + ring_b;
  L.harena = L.hist + (int64_t)hist_scores * 4;
  L.rev = L.harena + ((hist_words + 3) & ~(int64_t)3);
  L.cig = L.rev + ((int64_t)seq_len_sum + 48) / 4 + 8;
  L.words = L.cig + ((int64_t)2 * seq_len_sum + 16) / 4 + 8;
  L.words = (L.words + 63) & ~(int64_t)63;
  return L;
}

bool needs_general(const AlignParams& P);
cudaError_t launch_biwfa(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t launch_unialign(const AlignParams& P, int metric_class, int blocks, size_t smem,
                            cudaStream_t st);
int occupancy_blocks_per_sm(const AlignParams& P, int metric_class, size_t smem);

}  // namespace wfab
