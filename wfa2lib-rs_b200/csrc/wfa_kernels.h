// wfa_kernels.h -- kernel launchers used by the host side.
#pragma once
#include <cuda_runtime.h>

#include "wfa_common.h"

namespace wfab {

constexpr int kWarpsPerBlock = 4;
constexpr int kMinBlocksPerSM = 6;  // register budget: 65536 / (6 * 128) = 85 per thread
constexpr int kDescBytes = 32;      // sizeof(WfD)
constexpr int kBiFrameBytes = 64 * 7 * 4;  // kBiMaxDepth BiFrames (the BiWFA recursion's stack)

// Per-block dynamic shared memory of the unidirectional kernel: descriptor
// rings, staged sequences and (optionally) ring cells, each as one slice per
// lane group (`groups` groups per block).
struct SmemLayout {
  size_t desc_bytes, seq_bytes, ring_bytes;  // per group
  size_t desc_off, seq_off, ring_off, total;  // per block
};
#if defined(__CUDACC__)
__host__ __device__
#endif
inline SmemLayout smem_layout(int desc_depth, int nc, int cell_slots, int ring_wmax, int seq_words,
                              int groups) {
  SmemLayout L;
  L.desc_bytes = (size_t)desc_depth * nc * kDescBytes;
  L.seq_bytes = (size_t)2 * seq_words * 4;
  L.ring_bytes = (size_t)cell_slots * ring_wmax * 4;
  L.desc_off = 0;
  L.seq_off = L.desc_off + (size_t)groups * L.desc_bytes;
  L.ring_off = L.seq_off + (size_t)groups * L.seq_bytes;
  L.total = L.ring_off + (size_t)groups * L.ring_bytes;
  return L;
}

// Cell slots of a lane group's ring: the compact ring's, or one per score and
// component.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int cell_slots(const AlignParams& P, int nc) {
  return P.ring_slots > 0 ? P.ring_slots : P.scope * nc;
}

// Words at the start of a lane group's scratch slice taken by ring cells:
// the whole ring when its cells are not in shared memory, else the spill
// ring of the compact layout (if any).  A multiple of 4 (16-byte records
// follow).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int64_t slice_ring_words(const AlignParams& P, int nc) {
  const int64_t slots = cell_slots(P, nc);
  int64_t w = P.ring_smem ? (P.ring_slots > 0 ? slots * P.wspill : 0) : slots * P.wmax;
  if (P.piggyback && P.compute_alignment && !P.ring_smem) w *= 3;  // offsets, pcigars, block indices
  return (w + 3) & ~(int64_t)3;
}

// Words of a lane group's med/low backtrace buffer (after the dominance
// array): blocks (2 words each), initial positions (2 words each), then the
// compaction bitmap and its word counts.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int64_t slice_bt_words(const AlignParams& P) {
  if (!(P.piggyback && P.compute_alignment)) return 0;
  const int64_t marks = 2 * (((int64_t)P.bt_cap + 31) / 32);
  return (2 * (int64_t)P.bt_cap + 2 * (int64_t)P.bt_init_cap + marks + 3) & ~(int64_t)3;
}

// BiWFA per-group scratch slice (int32 word offsets).  seq_len_sum is the
// longest n + m of the launch (sizes the reversed sequences and the base
// CIGAR); idc_rows: the forward and reverse rings' extra rows
// (bi_idc_rows).
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
                          int64_t hist_words, int seq_len_sum, int idc_rows) {
  BiLayout L;
  const int64_t ring = (((int64_t)scope * nc + idc_rows) * wmax + 3) & ~(int64_t)3;
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

// Cost ordering of a batch (wfa_order.cu): order_count computes each pair's
// 4-mer profile distance key, the key histogram (kOrderBins bins, highest
// key first), the longest n + m and the longest sequence (two words at
// max_len_sum); order_scatter writes the pair indices
// in bin order into a list for the kernel's work queue.  hist and fill
// (kOrderBins ints each) start zeroed.
constexpr int kOrderBins = 1024;
size_t order_count_smem();
cudaError_t launch_order_count(const uint8_t* seq, int packed, const int64_t* p_off, const int32_t* p_len,
                               const int64_t* t_off, const int32_t* t_len, int64_t n, int num_sms,
                               int32_t* max_len_sum, uint16_t* keys, int32_t* hist, cudaStream_t st);
cudaError_t launch_order_scatter(const uint16_t* keys, int64_t n, const int32_t* hist, int32_t* fill,
                                 int64_t* list, int num_sms, cudaStream_t st);
// Both in one cooperative launch where the device supports it (else the two
// launches); *launches: how many were made.
cudaError_t launch_order(const uint8_t* seq, int packed, const int64_t* p_off, const int32_t* p_len,
                         const int64_t* t_off, const int32_t* t_len, int64_t n, int num_sms, int32_t* max_len_sum,
                         uint16_t* keys, int32_t* hist, int32_t* fill, int64_t* list, cudaStream_t st,
                         int* launches);

bool needs_general(const AlignParams& P);
// BiWFA: lanes per pair 32 (a warp) or 128, 256, 512 (a team of warps; the
// lean kernels only -- the kernels with heuristic support take 32 whatever
// is asked); blocks of bi_block_threads(lanes) threads, bi_groups_per_block
// pairs at a time, bi_smem_bytes of dynamic shared memory.
constexpr int bi_block_threads(int lanes) { return lanes > 128 ? lanes : 128; }
inline int bi_lanes_built(int lanes, bool gen) {
  return gen ? 32 : (lanes == 128 || lanes == 256 || lanes == 512) ? lanes : 32;
}
inline int bi_groups_per_block(int lanes) { return bi_block_threads(lanes) / lanes; }
inline size_t bi_smem_bytes(int lanes, int scope, int nc) {
  return (size_t)bi_groups_per_block(lanes) * (3 * (size_t)scope * nc * kDescBytes + kBiFrameBytes);
}
cudaError_t launch_biwfa(const AlignParams& P, int cls, int lanes, int blocks, size_t smem, cudaStream_t st);
int occupancy_biwfa(const AlignParams& P, int cls, int lanes, size_t smem);
// Lanes per pair: 4, 8, 16 or 32 (32 / lanes pairs per warp).
cudaError_t launch_unialign(const AlignParams& P, int metric_class, int lanes, int blocks, size_t smem,
                            cudaStream_t st);
int occupancy_blocks_per_sm(const AlignParams& P, int metric_class, int lanes, size_t smem);

}  // namespace wfab
