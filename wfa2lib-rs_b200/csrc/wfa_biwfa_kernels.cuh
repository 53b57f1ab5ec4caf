// wfa_biwfa_kernels.cuh -- the persistent BiWFA kernel for sm_100a, compiled
// once per sequence encoding and heuristic support (wfa_biwfa_{packed,ascii}
// {,_gen}.cu) so the four parts build in parallel beside the unidirectional
// kernels.  GEN = false is the lean instantiation (no heuristic).
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#include "wfa_biwfa.cuh"
#include "wfa_kernels.h"

namespace wfab {

static_assert(kBiMaxDepth * sizeof(BiFrame) == kBiFrameBytes, "frame stack size");
static_assert(sizeof(WfD) == kDescBytes, "descriptor size");

// ---------------------------------------------------------------------------
// BiWFA: one lane group per pair, a warp (LW = 32) or a team of LW / 32 warps
// (LW = 128, 256, 512); blocks of bi_block_threads(LW) threads.  Per group,
// shared memory holds the three descriptor rings (forward, reverse, base)
// and the recursion's frame stack; the scratch slice holds their cells, the
// base case's history, the reversed sequences and the base CIGAR.
// ---------------------------------------------------------------------------
template <int LW>
constexpr int bi_min_blocks() {
  // 255 registers for a warp per pair (its aligner state does not fit 128
  // without spills); teams are held to 128 so that 16 warps fit an SM.
  return LW == 32 ? 2 : 512 / bi_block_threads(LW);
}

template <int CLS, int ENC, bool GEN, int LW>
__global__ void __launch_bounds__(bi_block_threads(LW), bi_min_blocks<LW>()) biwfa_kernel(const AlignParams P) {
  extern __shared__ __align__(16) uint8_t smem[];
  using G = Lanes<LW>;
  constexpr int kGroups = bi_block_threads(LW) / LW;
  static_assert(LW <= 32 || kGroups == 1, "a team is a whole block");
  __shared__ unsigned long long next_pair[kGroups];
  const int grp = threadIdx.x / LW;
  const int lane = G::lane();
  const int64_t ggrp = (int64_t)blockIdx.x * kGroups + grp;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const BiLayout L = bi_layout(P.scope, NC, P.wmax, P.wmax_base, P.hist_scores, P.hist_words, P.max_len_sum,
                               bi_idc_rows(NC, P.e1, P.e2));
  WfD* desc = reinterpret_cast<WfD*>(smem) + (size_t)grp * 3 * P.scope * NC;
  BiFrame* frames = reinterpret_cast<BiFrame*>(smem + (size_t)kGroups * 3 * P.scope * NC * sizeof(WfD)) +
                    (size_t)grp * kBiMaxDepth;
  int32_t* slice = P.scratch + ggrp * P.warp_words;
  BiWorkspace bw;
  bw.fwd = Workspace{desc, slice + L.ring_f, nullptr, nullptr};
  bw.rev = Workspace{desc + P.scope * NC, slice + L.ring_r, nullptr, nullptr};
  bw.base = Workspace{desc + 2 * P.scope * NC, slice + L.ring_b,
                      reinterpret_cast<int4*>(slice + L.hist), slice + L.harena};
  bw.rev_seq = reinterpret_cast<uint8_t*>(slice + L.rev);
  bw.cig_tmp = reinterpret_cast<uint8_t*>(slice + L.cig);
  bw.frames = frames;
  for (;;) {
    if (lane == 0) next_pair[grp] = atomicAdd(P.work_counter, 1ull);
    G::sync();
    const unsigned long long idx = next_pair[grp];
    if (idx >= (unsigned long long)P.num_pairs) break;
    const int64_t pair = P.pair_list ? P.pair_list[idx] : (int64_t)idx;
    const int n = P.p_len[pair], m = P.t_len[pair];
    bool retry;
    if (ENC == WFA_SEQ_PACKED2) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(P.seq);
      SeqPacked sp{w + P.p_off[pair], n, (n + 15) >> 4};
      SeqPacked st{w + P.t_off[pair], m, (m + 15) >> 4};
      uint32_t* rp = reinterpret_cast<uint32_t*>(bw.rev_seq);
      uint32_t* rt = rp + ((n + 15) >> 4) + 1;
      reverse_into<LW>(sp, rp);
      reverse_into<LW>(st, rt);
      G::sync();
      SeqPacked rsp{rp, n, (n + 15) >> 4};
      SeqPacked rst{rt, m, (m + 15) >> 4};
      retry = biwfa_one<CLS, SeqPacked, GEN, LW>(P, bw, pair, sp, st, rsp, rst);
    } else {
      SeqAscii sp{P.seq + P.p_off[pair], n};
      SeqAscii st{P.seq + P.t_off[pair], m};
      uint8_t* rp = bw.rev_seq;
      uint8_t* rt = rp + ((n + 16) & ~15);
      reverse_into<LW>(sp, rp);
      reverse_into<LW>(st, rt);
      G::sync();
      SeqAscii rsp{rp, n};
      SeqAscii rst{rt, m};
      retry = biwfa_one<CLS, SeqAscii, GEN, LW>(P, bw, pair, sp, st, rsp, rst);
    }
    if (retry && lane == 0) {
      P.results[pair].status = kStatusRetry;
      atomicAdd(P.retry_count, 1);
    }
    G::sync();  // every lane has read next_pair before lane 0 refills it
  }
}

template <int CLS, int ENC, bool GEN, int LW>
static cudaError_t launch_bi_t(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  auto k = biwfa_kernel<CLS, ENC, GEN, LW>;
  // Dynamic shared memory already allowed for k; only ever raised, under a
  // lock (handles on several host threads launch the same kernels).
  static size_t configured = 0;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (smem > configured) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      configured = smem;
    }
  }
  k<<<blocks, bi_block_threads(LW), smem, st>>>(P);
  return cudaGetLastError();
}

// The launches of one encoding (ENC: wfa_seq_format_t), heuristic support
// and lane-group width, one translation unit each (wfa_biwfa_*.cu), so that
// they build in parallel.
template <int ENC, bool GEN, int LW>
cudaError_t launch_biwfa_lw(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  switch (cls) {
    case kEditClass: return launch_bi_t<kEditClass, ENC, GEN, LW>(P, blocks, smem, st);
    case kLinearClass: return launch_bi_t<kLinearClass, ENC, GEN, LW>(P, blocks, smem, st);
    case kAffineClass: return launch_bi_t<kAffineClass, ENC, GEN, LW>(P, blocks, smem, st);
    default: return launch_bi_t<kAffine2pClass, ENC, GEN, LW>(P, blocks, smem, st);
  }
}

// Resident blocks per SM of a launch (0 if the query fails).
template <int ENC, bool GEN, int LW>
int occupancy_biwfa_lw(int cls, size_t smem) {
  int nb = 0;
  cudaError_t e;
  // Loads the kernel if it is not yet (see occ_t in wfa_unialign.cuh).
  cudaFuncAttributes fa;
  const void* fk = cls == kEditClass     ? (const void*)biwfa_kernel<kEditClass, ENC, GEN, LW>
                   : cls == kLinearClass ? (const void*)biwfa_kernel<kLinearClass, ENC, GEN, LW>
                   : cls == kAffineClass ? (const void*)biwfa_kernel<kAffineClass, ENC, GEN, LW>
                                         : (const void*)biwfa_kernel<kAffine2pClass, ENC, GEN, LW>;
  if (cudaFuncGetAttributes(&fa, fk) != cudaSuccess) cudaGetLastError();
  switch (cls) {
    case kEditClass:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, biwfa_kernel<kEditClass, ENC, GEN, LW>,
                                                        bi_block_threads(LW), smem);
      break;
    case kLinearClass:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, biwfa_kernel<kLinearClass, ENC, GEN, LW>,
                                                        bi_block_threads(LW), smem);
      break;
    case kAffineClass:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, biwfa_kernel<kAffineClass, ENC, GEN, LW>,
                                                        bi_block_threads(LW), smem);
      break;
    default:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, biwfa_kernel<kAffine2pClass, ENC, GEN, LW>,
                                                        bi_block_threads(LW), smem);
  }
  return e == cudaSuccess ? nb : 0;
}

#define WFA_BIWFA_INSTANCE(ENC, GEN, LW)                                                              \
  template cudaError_t launch_biwfa_lw<ENC, GEN, LW>(const AlignParams&, int, int, size_t, cudaStream_t); \
  template int occupancy_biwfa_lw<ENC, GEN, LW>(int, size_t);
#define WFA_BIWFA_EXTERN(ENC, GEN, LW)                                                                       \
  extern template cudaError_t launch_biwfa_lw<ENC, GEN, LW>(const AlignParams&, int, int, size_t, cudaStream_t); \
  extern template int occupancy_biwfa_lw<ENC, GEN, LW>(int, size_t);

}  // namespace wfab
