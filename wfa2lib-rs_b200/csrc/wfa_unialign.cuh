// wfa_unialign.cuh -- the persistent unidirectional-WFA kernel for sm_100a
// and its launch helpers, instantiated per lane-group width in
// wfa_kernels_*.cu (translation units that build in parallel).
//
// Launch shape: blocks of kWarpsPerBlock warps, grid sized to the SM count
// times the resident blocks per SM.  Each warp pulls pair indices from a
// device counter (work queue), so pairs of uneven length and score balance
// across the machine.  Per warp, shared memory holds the wavefront
// descriptor ring, the pair's sequences (when short enough) and, when the
// ring is narrow enough, its cells; otherwise cells live in the warp's slice
// of the scratch buffer, as does the M history of CIGAR mode.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "wfa_align.cuh"
#include "wfa_kernels.h"

namespace wfab {

// Register budget: the lean instantiations of the smaller metrics fit 80
// registers (6 blocks = 24 warps per SM); the general and two-piece ones keep
// 128 (4 blocks) rather than spill.
// The med/low instantiation carries three arrays per cell and the backtrace
// buffer: 2 blocks per SM (up to 255 registers) rather than spill.
// With 4 lanes per pair a block's 32 rings in shared memory already hold an
// SM to 5 blocks, so that width gets the registers of 5 (96) instead of
// spilling to fit a sixth block that could not be resident.
template <int CLS, bool GEN, bool PB = false, int LW = 32>
constexpr int min_blocks() {
  return PB ? 2 : (GEN || CLS == kAffine2pClass) ? 4 : LW == 4 ? 5 : kMinBlocksPerSM;
}

// The sequences of pair `pair`, staged in the group's shared memory (2 x sw
// words) when both fit, else read from device memory.
template <int LW>
WFA_D void pair_seqs(const AlignParams& P, int64_t pair, uint32_t* sseq, int sw, int lane, SeqPacked& sp,
                     SeqPacked& st) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(P.seq);
  sp = SeqPacked{w + P.p_off[pair], P.p_len[pair], (P.p_len[pair] + 15) >> 4};
  st = SeqPacked{w + P.t_off[pair], P.t_len[pair], (P.t_len[pair] + 15) >> 4};
  if (sp.nw <= sw && st.nw <= sw) {
    for (int i = lane; i < sp.nw; i += LW) sseq[i] = sp.w[i];
    for (int i = lane; i < st.nw; i += LW) sseq[sw + i] = st.w[i];
    Lanes<LW>::sync();
    sp.w = sseq;
    st.w = sseq + sw;
  }
}
template <int LW>
WFA_D void pair_seqs(const AlignParams& P, int64_t pair, uint32_t* sseq, int sw, int lane, SeqAscii& sp,
                     SeqAscii& st) {
  sp = SeqAscii{P.seq + P.p_off[pair], P.p_len[pair]};
  st = SeqAscii{P.seq + P.t_off[pair], P.t_len[pair]};
  const uintptr_t pa = (uintptr_t)sp.p, ta = (uintptr_t)st.p;
  const int pw = sp.len > 0 ? (int)(((pa + sp.len + 3) & ~(uintptr_t)3) - (pa & ~(uintptr_t)3)) / 4 : 0;
  const int tw = st.len > 0 ? (int)(((ta + st.len + 3) & ~(uintptr_t)3) - (ta & ~(uintptr_t)3)) / 4 : 0;
  if (pw <= sw && tw <= sw) {
    const uint32_t* pg = reinterpret_cast<const uint32_t*>(pa & ~(uintptr_t)3);
    const uint32_t* tg = reinterpret_cast<const uint32_t*>(ta & ~(uintptr_t)3);
    for (int i = lane; i < pw; i += LW) sseq[i] = pg[i];
    for (int i = lane; i < tw; i += LW) sseq[sw + i] = tg[i];
    Lanes<LW>::sync();
    sp.p = reinterpret_cast<const uint8_t*>(sseq) + (pa & 3);
    st.p = reinterpret_cast<const uint8_t*>(sseq + sw) + (ta & 3);
  }
}

// Next pair index of the launch's work queue for a lane group (lane 0 takes
// it, the group shares it); -1 when the queue is empty.
template <int LW>
WFA_D int64_t next_pair(const AlignParams& P, int lane) {
  unsigned long long idx = 0;
  if (lane == 0) idx = atomicAdd(P.work_counter, 1ull);
  idx = __shfl_sync(Lanes<LW>::mask(), idx, 0, LW);
  if (idx >= (unsigned long long)P.num_pairs) return -1;
  return P.pair_list ? P.pair_list[idx] : (int64_t)idx;
}

template <int LW>
WFA_D void mark_retry(const AlignParams& P, int64_t pair, int lane) {
  if (lane == 0) {
    P.results[pair].status = kStatusRetry;
    atomicAdd(P.retry_count, 1);
  }
}

template <int CLS, int ENC, bool GEN, int LW, bool PB = false>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (min_blocks<CLS, GEN, PB, LW>()))
    unialign_kernel(const AlignParams P) {
  extern __shared__ __align__(16) uint8_t smem[];
  constexpr int kGroups = kWarpsPerBlock * 32 / LW;  // lane groups (pairs in flight) per block
  using G = Lanes<LW>;
  using S = typename std::conditional<ENC == WFA_SEQ_PACKED2, SeqPacked, SeqAscii>::type;
  const int gib = threadIdx.x / LW;
  const int lane = G::lane();
  const int64_t ggroup = (int64_t)blockIdx.x * kGroups + gib;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const int slots = cell_slots(P, NC);
  const SmemLayout L = smem_layout(P.desc_depth ? P.desc_depth : P.scope, NC, slots, P.ring_smem ? P.wmax : 0,
                                   P.seq_smem_words, kGroups);
  Workspace ws;
  ws.ring = reinterpret_cast<WfD*>(smem + L.desc_off + (size_t)gib * L.desc_bytes);
  uint32_t* sseq = reinterpret_cast<uint32_t*>(smem + L.seq_off + (size_t)gib * L.seq_bytes);
  int32_t* slice = P.scratch + ggroup * P.warp_words;
  const int64_t ring_words = slice_ring_words(P, NC);
  ws.ringv = P.ring_smem ? reinterpret_cast<int32_t*>(smem + L.ring_off + (size_t)gib * L.ring_bytes)
                         : slice;
  ws.ringg = P.ring_smem && P.ring_slots > 0 && P.wspill > 0 ? slice : nullptr;
  ws.hist = reinterpret_cast<int4*>(slice + ring_words);
  ws.harena = slice + ring_words + (int64_t)P.hist_scores * 4;
  ws.dom = P.dom_words ? ws.harena + P.hist_words : nullptr;
  int32_t* btb = ws.harena + ((P.hist_words + P.dom_words + 3) & ~(int64_t)3);  // 16-byte aligned
  ws.bt = reinterpret_cast<uint2*>(btb);
  ws.btinit = reinterpret_cast<int2*>(btb + 2 * (int64_t)P.bt_cap);
  ws.btmark = reinterpret_cast<uint32_t*>(btb + 2 * (int64_t)P.bt_cap + 2 * (int64_t)P.bt_init_cap);
  const int sw = P.seq_smem_words;
  // Each lane group pulls pairs from the launch's work queue.  The groups of
  // a warp run their pairs side by side (lockstep per pair: the warp's
  // reconvergence points are the ends of the pairs' loops); a group that is
  // done first waits for the others, and all then take their next pairs.
  for (;;) {
    const int64_t pair = next_pair<LW>(P, lane);
    if (pair < 0) break;
    S sp, st;
    pair_seqs<LW>(P, pair, sseq, sw, lane, sp, st);
    if (align_one<CLS, S, GEN, LW, PB>(P, ws, pair, sp, st)) mark_retry<LW>(P, pair, lane);
    G::sync();
  }
}

// Allows the kernel `smem` bytes of dynamic shared memory.  The allowance
// is only ever raised, under a lock: handles on several host threads launch
// the same kernels, and lowering it under another thread's launch would make
// that launch fail.
template <int CLS, int ENC, bool GEN, int LW, bool PB = false>
static cudaError_t allow_smem(size_t smem) {
  static size_t configured = 0;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(unialign_kernel<CLS, ENC, GEN, LW, PB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = smem;
  }
  return cudaSuccess;
}

template <int CLS, int ENC, bool GEN, int LW, bool PB = false>
static cudaError_t launch_t(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  auto k = unialign_kernel<CLS, ENC, GEN, LW, PB>;
  cudaError_t e = allow_smem<CLS, ENC, GEN, LW, PB>(smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, kWarpsPerBlock * 32, smem, st>>>(P);
  return cudaGetLastError();
}

template <int CLS, int ENC, bool GEN, int LW, bool PB = false>
static int occ_t(size_t smem) {
  int nb = 0;
  auto k = unialign_kernel<CLS, ENC, GEN, LW, PB>;
  // Loads the kernel if it is not yet (the server loads every kernel this
  // way before its resident lane starts).
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) cudaGetLastError();
  if (allow_smem<CLS, ENC, GEN, LW, PB>(smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kWarpsPerBlock * 32, smem) != cudaSuccess) {
    cudaGetLastError();
    nb = 1;
  }
  return nb < 1 ? 1 : nb;
}

}  // namespace wfab
