// wfa_kernels.cu -- the persistent unidirectional-WFA kernel for sm_100a.
//
// Launch shape: blocks of kWarpsPerBlock warps, grid sized to the SM count
// times the resident blocks per SM.  Each warp pulls pair indices from a
// device counter (work queue), so pairs of uneven length and score balance
// across the machine.  Per warp, shared memory holds the wavefront
// descriptor ring, the pair's sequences (when short enough) and, when the
// ring is narrow enough, its cells; otherwise cells live in the warp's slice
// of the scratch buffer, as does the M history of CIGAR mode.
#include <cuda_runtime.h>

#include <mutex>

#include "wfa_align.cuh"
#include "wfa_kernels.h"

namespace wfab {

// Register budget: the lean instantiations of the smaller metrics fit 80
// registers (6 blocks = 24 warps per SM); the general and two-piece ones keep
// 128 (4 blocks) rather than spill.
template <int CLS, bool GEN>
constexpr int min_blocks() { return (GEN || CLS == kAffine2pClass) ? 4 : kMinBlocksPerSM; }

template <int CLS, int ENC, bool GEN>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (min_blocks<CLS, GEN>()))
    unialign_kernel(const AlignParams P) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const SmemLayout L = smem_layout(P.scope, NC, P.ring_smem ? P.wmax : 0, P.seq_smem_words);
  Workspace ws;
  ws.ring = reinterpret_cast<WfD*>(smem + L.desc_off + (size_t)wib * L.desc_bytes);
  uint32_t* sseq = reinterpret_cast<uint32_t*>(smem + L.seq_off + (size_t)wib * L.seq_bytes);
  int32_t* slice = P.scratch + gwarp * P.warp_words;
  int64_t ring_words = P.ring_smem ? 0 : (((int64_t)P.scope * NC * P.wmax + 3) & ~(int64_t)3);
  ws.ringv = P.ring_smem ? reinterpret_cast<int32_t*>(smem + L.ring_off + (size_t)wib * L.ring_bytes)
                         : slice;
  ws.hist = reinterpret_cast<int4*>(slice + ring_words);
  ws.harena = slice + ring_words + (int64_t)P.hist_scores * 4;
  ws.dom = P.dom_words ? ws.harena + P.hist_words : nullptr;
  const int sw = P.seq_smem_words;
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
      // Stage both sequences in shared memory when they fit.
      if (sp.nw <= sw && st.nw <= sw) {
        for (int i = lane; i < sp.nw; i += 32) sseq[i] = sp.w[i];
        for (int i = lane; i < st.nw; i += 32) sseq[sw + i] = st.w[i];
        __syncwarp();
        sp.w = sseq;
        st.w = sseq + sw;
      }
      retry = align_one<CLS, SeqPacked, GEN>(P, ws, pair, sp, st);
    } else {
      SeqAscii sp{P.seq + P.p_off[pair], P.p_len[pair]};
      SeqAscii st{P.seq + P.t_off[pair], P.t_len[pair]};
      const uintptr_t pa = (uintptr_t)sp.p, ta = (uintptr_t)st.p;
      const int pw = sp.len > 0 ? (int)(((pa + sp.len + 3) & ~(uintptr_t)3) - (pa & ~(uintptr_t)3)) / 4 : 0;
      const int tw = st.len > 0 ? (int)(((ta + st.len + 3) & ~(uintptr_t)3) - (ta & ~(uintptr_t)3)) / 4 : 0;
      if (pw <= sw && tw <= sw) {
        const uint32_t* pg = reinterpret_cast<const uint32_t*>(pa & ~(uintptr_t)3);
        const uint32_t* tg = reinterpret_cast<const uint32_t*>(ta & ~(uintptr_t)3);
        for (int i = lane; i < pw; i += 32) sseq[i] = pg[i];
        for (int i = lane; i < tw; i += 32) sseq[sw + i] = tg[i];
        __syncwarp();
        sp.p = reinterpret_cast<const uint8_t*>(sseq) + (pa & 3);
        st.p = reinterpret_cast<const uint8_t*>(sseq + sw) + (ta & 3);
      }
      retry = align_one<CLS, SeqAscii, GEN>(P, ws, pair, sp, st);
    }
    if (retry && lane == 0) {
      P.results[pair].status = kStatusRetry;
      atomicAdd(P.retry_count, 1);
    }
    __syncwarp();
  }
}

// Allows the kernel `smem` bytes of dynamic shared memory.  The allowance
// is only ever raised, under a lock: handles on several host threads launch
// the same kernels, and lowering it under another thread's launch would make
// that launch fail.
template <int CLS, int ENC, bool GEN>
static cudaError_t allow_smem(size_t smem) {
  static size_t configured = 0;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(unialign_kernel<CLS, ENC, GEN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = smem;
  }
  return cudaSuccess;
}

template <int CLS, int ENC, bool GEN>
static cudaError_t launch_t(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  auto k = unialign_kernel<CLS, ENC, GEN>;
  cudaError_t e = allow_smem<CLS, ENC, GEN>(smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, kWarpsPerBlock * 32, smem, st>>>(P);
  return cudaGetLastError();
}

template <int CLS, bool GEN>
static cudaError_t launch_c(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  return P.format == WFA_SEQ_PACKED2 ? launch_t<CLS, 1, GEN>(P, blocks, smem, st)
                                     : launch_t<CLS, 0, GEN>(P, blocks, smem, st);
}

template <bool GEN>
static cudaError_t launch_g(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  switch (cls) {
    case kEditClass: return launch_c<kEditClass, GEN>(P, blocks, smem, st);
    case kLinearClass: return launch_c<kLinearClass, GEN>(P, blocks, smem, st);
    case kAffineClass: return launch_c<kAffineClass, GEN>(P, blocks, smem, st);
    default: return launch_c<kAffine2pClass, GEN>(P, blocks, smem, st);
  }
}

// The lean instantiation runs end-to-end high-memory alignments without a
// heuristic; everything else (ends-free, heuristics, the med/low piggyback
// backtrace) runs the general one.
bool needs_general(const AlignParams& P) {
  return P.span != WFA_SPAN_END2END || P.hkind != WFA_HEURISTIC_NONE || P.piggyback;
}

cudaError_t launch_unialign(const AlignParams& P, int metric_class, int blocks, size_t smem,
                            cudaStream_t st) {
  return needs_general(P) ? launch_g<true>(P, metric_class, blocks, smem, st)
                          : launch_g<false>(P, metric_class, blocks, smem, st);
}

template <int CLS, int ENC, bool GEN>
static int occ_t(size_t smem) {
  int nb = 0;
  auto k = unialign_kernel<CLS, ENC, GEN>;
  if (allow_smem<CLS, ENC, GEN>(smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kWarpsPerBlock * 32, smem) != cudaSuccess) {
    cudaGetLastError();
    nb = 1;
  }
  return nb < 1 ? 1 : nb;
}

template <bool GEN>
static int occ_g(int cls, bool packed, size_t smem) {
  switch (cls) {
    case kEditClass: return packed ? occ_t<kEditClass, 1, GEN>(smem) : occ_t<kEditClass, 0, GEN>(smem);
    case kLinearClass: return packed ? occ_t<kLinearClass, 1, GEN>(smem) : occ_t<kLinearClass, 0, GEN>(smem);
    case kAffineClass: return packed ? occ_t<kAffineClass, 1, GEN>(smem) : occ_t<kAffineClass, 0, GEN>(smem);
    default: return packed ? occ_t<kAffine2pClass, 1, GEN>(smem) : occ_t<kAffine2pClass, 0, GEN>(smem);
  }
}

int occupancy_blocks_per_sm(const AlignParams& P, int metric_class, size_t smem) {
  const bool packed = P.format == WFA_SEQ_PACKED2;
  return needs_general(P) ? occ_g<true>(metric_class, packed, smem)
                          : occ_g<false>(metric_class, packed, smem);
}

}  // namespace wfab
