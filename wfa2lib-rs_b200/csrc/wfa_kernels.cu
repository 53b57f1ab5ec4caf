// wfa_kernels.cu -- the persistent unidirectional-WFA kernel for sm_100a.
//
// Launch shape: blocks of kWarpsPerBlock warps, grid sized to the SM count
// times the resident blocks per SM.  Each warp pulls pair indices from a
// device counter (work queue), so pairs of uneven length and score balance
// across the machine; its wavefront descriptors live in shared memory and its
// wavefront cells in a private slice of the scratch buffer (ring slots, plus
// the M history in CIGAR mode).
#include <cuda_runtime.h>

#include "wfa_align.cuh"
#include "wfa_kernels.h"

namespace wfab {

template <int CLS, int ENC>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    unialign_kernel(const AlignParams P) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  Workspace ws;
  ws.ring = reinterpret_cast<WfD*>(smem) + (int64_t)wib * P.scope * NC;
  int32_t* slice = P.scratch + gwarp * P.warp_words;
  ws.ringv = slice;
  int64_t ring_words = (int64_t)P.scope * NC * P.wmax;
  ring_words = (ring_words + 3) & ~(int64_t)3;
  ws.hist = reinterpret_cast<int4*>(slice + ring_words);
  ws.harena = slice + ring_words + (int64_t)P.hist_scores * 4;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(P.work_counter, 1ull);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= (unsigned long long)P.num_pairs) break;
    const int64_t pair = P.pair_list ? P.pair_list[idx] : (int64_t)idx;
    bool retry;
    if (ENC == WFA_SEQ_PACKED2) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(P.seq);
      SeqPacked sp{w + P.p_off[pair], P.p_len[pair], (P.p_len[pair] + 15) >> 4};
      SeqPacked st{w + P.t_off[pair], P.t_len[pair], (P.t_len[pair] + 15) >> 4};
      retry = align_one<CLS, SeqPacked>(P, ws, pair, sp, st);
    } else {
      SeqAscii sp{P.seq + P.p_off[pair], P.p_len[pair]};
      SeqAscii st{P.seq + P.t_off[pair], P.t_len[pair]};
      retry = align_one<CLS, SeqAscii>(P, ws, pair, sp, st);
    }
    if (retry && lane == 0) {
      P.results[pair].status = kStatusRetry;
      atomicAdd(P.retry_count, 1);
    }
    __syncwarp();
  }
}

template <int CLS, int ENC>
static cudaError_t launch_t(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  auto k = unialign_kernel<CLS, ENC>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, kWarpsPerBlock * 32, smem, st>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_unialign(const AlignParams& P, int metric_class, int blocks, size_t smem,
                            cudaStream_t st) {
  const bool packed = P.format == WFA_SEQ_PACKED2;
  switch (metric_class) {
    case kEditClass:
      return packed ? launch_t<kEditClass, 1>(P, blocks, smem, st) : launch_t<kEditClass, 0>(P, blocks, smem, st);
    case kLinearClass:
      return packed ? launch_t<kLinearClass, 1>(P, blocks, smem, st) : launch_t<kLinearClass, 0>(P, blocks, smem, st);
    case kAffineClass:
      return packed ? launch_t<kAffineClass, 1>(P, blocks, smem, st) : launch_t<kAffineClass, 0>(P, blocks, smem, st);
    default:
      return packed ? launch_t<kAffine2pClass, 1>(P, blocks, smem, st)
                    : launch_t<kAffine2pClass, 0>(P, blocks, smem, st);
  }
}

int occupancy_blocks_per_sm(int metric_class, bool packed, size_t smem) {
  int nb = 0;
  cudaError_t e = cudaSuccess;
#define OCC(C, E) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, unialign_kernel<C, E>, kWarpsPerBlock * 32, smem)
  switch (metric_class) {
    case kEditClass: if (packed) OCC(kEditClass, 1); else OCC(kEditClass, 0); break;
    case kLinearClass: if (packed) OCC(kLinearClass, 1); else OCC(kLinearClass, 0); break;
    case kAffineClass: if (packed) OCC(kAffineClass, 1); else OCC(kAffineClass, 0); break;
    default: if (packed) OCC(kAffine2pClass, 1); else OCC(kAffine2pClass, 0); break;
  }
#undef OCC
  if (e != cudaSuccess || nb < 1) nb = 1;
  return nb;
}

}  // namespace wfab
