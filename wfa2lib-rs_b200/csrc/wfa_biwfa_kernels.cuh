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

// ---------------------------------------------------------------------------
// BiWFA: one warp per pair; per warp, shared memory holds the three
// descriptor rings (forward, reverse, base) and the scratch slice their cells,
// the base case's history, the reversed sequences and the base CIGAR.
// ---------------------------------------------------------------------------
template <int CLS, int ENC, bool GEN>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 2) biwfa_kernel(const AlignParams P) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const BiLayout L = bi_layout(P.scope, NC, P.wmax, P.wmax_base, P.hist_scores, P.hist_words, P.max_len_sum);
  WfD* desc = reinterpret_cast<WfD*>(smem) + (size_t)wib * 3 * P.scope * NC;
  int32_t* slice = P.scratch + gwarp * P.warp_words;
  BiWorkspace bw;
  bw.fwd = Workspace{desc, slice + L.ring_f, nullptr, nullptr};
  bw.rev = Workspace{desc + P.scope * NC, slice + L.ring_r, nullptr, nullptr};
  bw.base = Workspace{desc + 2 * P.scope * NC, slice + L.ring_b,
                      reinterpret_cast<int4*>(slice + L.hist), slice + L.harena};
  bw.rev_seq = reinterpret_cast<uint8_t*>(slice + L.rev);
  bw.cig_tmp = reinterpret_cast<uint8_t*>(slice + L.cig);
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(P.work_counter, 1ull);
    idx = __shfl_sync(0xffffffffu, idx, 0);
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
      reverse_into(sp, rp);
      reverse_into(st, rt);
      __syncwarp();
      SeqPacked rsp{rp, n, (n + 15) >> 4};
      SeqPacked rst{rt, m, (m + 15) >> 4};
      retry = biwfa_one<CLS, SeqPacked, GEN>(P, bw, pair, sp, st, rsp, rst);
    } else {
      SeqAscii sp{P.seq + P.p_off[pair], n};
      SeqAscii st{P.seq + P.t_off[pair], m};
      uint8_t* rp = bw.rev_seq;
      uint8_t* rt = rp + ((n + 16) & ~15);
      reverse_into(sp, rp);
      reverse_into(st, rt);
      __syncwarp();
      SeqAscii rsp{rp, n};
      SeqAscii rst{rt, m};
      retry = biwfa_one<CLS, SeqAscii, GEN>(P, bw, pair, sp, st, rsp, rst);
    }
    if (retry && lane == 0) {
      P.results[pair].status = kStatusRetry;
      atomicAdd(P.retry_count, 1);
    }
    __syncwarp();
  }
}

template <int CLS, int ENC, bool GEN>
static cudaError_t launch_bi_t(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  auto k = biwfa_kernel<CLS, ENC, GEN>;
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
  k<<<blocks, kWarpsPerBlock * 32, smem, st>>>(P);
  return cudaGetLastError();
}

// The launches of one encoding (ENC: wfa_seq_format_t) and heuristic support.
template <int ENC, bool GEN>
cudaError_t launch_biwfa_enc(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  switch (cls) {
    case kEditClass: return launch_bi_t<kEditClass, ENC, GEN>(P, blocks, smem, st);
    case kLinearClass: return launch_bi_t<kLinearClass, ENC, GEN>(P, blocks, smem, st);
    case kAffineClass: return launch_bi_t<kAffineClass, ENC, GEN>(P, blocks, smem, st);
    default: return launch_bi_t<kAffine2pClass, ENC, GEN>(P, blocks, smem, st);
  }
}

}  // namespace wfab
