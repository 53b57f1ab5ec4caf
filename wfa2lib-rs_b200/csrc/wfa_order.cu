// wfa_order.cu -- cost ordering of a batch for the lane-group kernel.
//
// The lane groups of a warp align their pairs side by side, and a warp is as
// slow as its costliest pair, so pairs of similar cost should share warps.
// The persistent kernel hands out pairs in list order, four consecutive
// entries to the four groups of a warp, so the list is ordered by an
// estimate of each pair's cost, highest first (which also starts the longest
// work first).  The estimate is the 4-mer profile distance of the two
// sequences, sum over the 256 4-mers x of |count_P(x) - count_T(x)|: every
// edit changes at most eight 4-mer counts, and on the short-read batch the
// distance follows the alignment score closely (correlation about 0.93).
// The order only decides which pairs run together; results do not depend
// on it.
#include <cooperative_groups.h>
#include <cub/block/block_scan.cuh>

#include <algorithm>

#include "wfa_kernels.h"

namespace wfab {

constexpr int kCountBlock = 128;   // threads (pairs in flight) per counting block
constexpr int kProfileBases = 4096;  // bases of each sequence the estimate reads
// (2-bit codes: packed input as stored; ASCII bytes by their bits 1-2, which
// tell A, C, G and T apart -- enough for an estimate.)

// Per pair: the longest n + m of the batch and its longest sequence
// (atomicMax into max_len_sum[0] and [1]),
// the estimate key (keys[i], at most kOrderBins - 1) and the batch's key
// histogram (bin kOrderBins - 1 - key, so that bins ascend as costs fall).
// Each thread profiles its own pairs in a column of shared memory: two
// 16-bit counters per word, biased by kBias so that the at most
// kProfileBases increments or decrements of a counter never carry into its
// neighbour, updated with atomic adds whose results are not used (no update
// waits for the previous one).
constexpr uint32_t kBias = 0x4000;
__device__ __forceinline__ void count_body(uint8_t* smem, const uint8_t* seq, int packed, const int64_t* p_off,
                                           const int32_t* p_len, const int64_t* t_off, const int32_t* t_len,
                                           int64_t n, int32_t* max_len_sum, uint16_t* keys, int32_t* hist) {
  uint32_t* prof = reinterpret_cast<uint32_t*>(smem);  // [128 word][kCountBlock]: 4-mers 2w, 2w+1
  int32_t* bins = reinterpret_cast<int32_t*>(smem + 128 * kCountBlock * 4);
  const int tid = threadIdx.x;
  constexpr uint32_t kBiased = kBias | (kBias << 16);
  for (int b = tid; b < kOrderBins; b += kCountBlock) bins[b] = 0;
  for (int x = 0; x < 128; ++x) prof[x * kCountBlock + tid] = kBiased;
  __syncthreads();
  int32_t mx = 0, ms = 0;
  for (int64_t i = (int64_t)blockIdx.x * kCountBlock + tid; i < n; i += (int64_t)gridDim.x * kCountBlock) {
    const int32_t pn = p_len[i], tn = t_len[i];
    mx = max(mx, pn + tn);
    ms = max(ms, max(pn, tn));
    for (int s = 0; s < 2; ++s) {
      const int64_t off = s == 0 ? p_off[i] : t_off[i];
      const int len = min(s == 0 ? pn : tn, kProfileBases);
      // +1 or -1 on the low or the high half (as 32-bit adds: neither half
      // ever wraps, so -1 never borrows from the other half)
      const uint32_t dlo = s == 0 ? 1u : 0xFFFFFFFFu, dhi = s == 0 ? 1u << 16 : 0xFFFF0000u;
      uint32_t km = 0;
      // Bases in chunks of 16: one 32-bit load of 2-bit codes (packed) or
      // 16 byte loads (ASCII), then the chunk's 4-mers from registers.
      for (int j0 = 0; j0 < len; j0 += 16) {
        uint32_t codes = 0;
        if (packed) {
          codes = reinterpret_cast<const uint32_t*>(seq)[off + (j0 >> 4)];
        } else {
          const int lim = min(16, len - j0);
          for (int b = 0; b < lim; ++b) codes |= (((uint32_t)seq[off + j0 + b] >> 1) & 3u) << (2 * b);
        }
        const int lim = min(16, len - j0);
#pragma unroll
        for (int b = 0; b < 16; ++b) {
          if (b < lim) {
            km = ((km << 2) | ((codes >> (2 * b)) & 3u)) & 0xFFu;
            if (j0 + b >= 3) atomicAdd(&prof[(km >> 1) * kCountBlock + tid], (km & 1) ? dhi : dlo);
          }
        }
      }
    }
    int32_t l1 = 0;
    for (int x = 0; x < 128; ++x) {
      const uint32_t w = prof[x * kCountBlock + tid];
      const int32_t lo = (int32_t)(w & 0xFFFFu) - (int32_t)kBias, hi = (int32_t)(w >> 16) - (int32_t)kBias;
      l1 += (lo < 0 ? -lo : lo) + (hi < 0 ? -hi : hi);
      prof[x * kCountBlock + tid] = kBiased;
    }
    const int key = min(l1, kOrderBins - 1);
    keys[i] = (uint16_t)key;
    atomicAdd(&bins[kOrderBins - 1 - key], 1);
  }
  mx = __reduce_max_sync(0xffffffffu, mx);
  ms = __reduce_max_sync(0xffffffffu, ms);
  if ((tid & 31) == 0) {
    atomicMax(max_len_sum, mx);
    atomicMax(max_len_sum + 1, ms);
  }
  __syncthreads();
  for (int b = tid; b < kOrderBins; b += kCountBlock)
    if (bins[b]) atomicAdd(&hist[b], bins[b]);
}

__global__ void __launch_bounds__(kCountBlock) order_count(const uint8_t* seq, int packed,
                                                            const int64_t* p_off, const int32_t* p_len,
                                                            const int64_t* t_off, const int32_t* t_len,
                                                            int64_t n, int32_t* max_len_sum,
                                                            uint16_t* keys, int32_t* hist) {
  extern __shared__ __align__(16) uint8_t smem[];
  count_body(smem, seq, packed, p_off, p_len, t_off, t_len, n, max_len_sum, keys, hist);
}

constexpr int kScatterBlock = 256, kScatterItems = 8;
constexpr int kScatterTile = kScatterBlock * kScatterItems;

// list[] = the pair indices 0..n-1 in ascending bin order (falling cost).
// Each block scans the histogram, then places a tile of BLOCK x ITEMS pairs
// at a time: ranks within the tile from shared-memory counters, one global
// reservation per (tile, bin) in fill[].
template <int BLOCK, int ITEMS>
struct ScatterSmem {
  typename cub::BlockScan<int32_t, BLOCK>::TempStorage scan;
  int32_t start[kOrderBins];   // exclusive scan of hist
  int32_t tcount[kOrderBins];  // this tile's pairs per bin, then their base
};
template <int BLOCK, int ITEMS>
__device__ __forceinline__ void scatter_body(ScatterSmem<BLOCK, ITEMS>& sm, const uint16_t* keys, int64_t n,
                                             const int32_t* hist, int32_t* fill, int64_t* list) {
  using Scan = cub::BlockScan<int32_t, BLOCK>;
  constexpr int kPer = kOrderBins / BLOCK;
  constexpr int kTile = BLOCK * ITEMS;
  int32_t v[kPer];
  for (int j = 0; j < kPer; ++j) v[j] = hist[threadIdx.x * kPer + j];
  Scan(sm.scan).ExclusiveSum(v, v);
  for (int j = 0; j < kPer; ++j) sm.start[threadIdx.x * kPer + j] = v[j];
  for (int64_t t0 = (int64_t)blockIdx.x * kTile; t0 < n; t0 += (int64_t)gridDim.x * kTile) {
    for (int b = threadIdx.x; b < kOrderBins; b += BLOCK) sm.tcount[b] = 0;
    __syncthreads();
    int32_t bin[ITEMS], rank[ITEMS];
    for (int k = 0; k < ITEMS; ++k) {
      const int64_t i = t0 + (int64_t)k * BLOCK + threadIdx.x;
      bin[k] = i < n ? kOrderBins - 1 - keys[i] : -1;
      rank[k] = bin[k] >= 0 ? atomicAdd(&sm.tcount[bin[k]], 1) : 0;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kOrderBins; b += BLOCK)
      if (sm.tcount[b]) sm.tcount[b] = sm.start[b] + atomicAdd(&fill[b], sm.tcount[b]);
    __syncthreads();
    for (int k = 0; k < ITEMS; ++k) {
      const int64_t i = t0 + (int64_t)k * BLOCK + threadIdx.x;
      if (bin[k] >= 0) list[sm.tcount[bin[k]] + rank[k]] = i;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScatterBlock) order_scatter(const uint16_t* keys, int64_t n,
                                                               const int32_t* hist, int32_t* fill,
                                                               int64_t* list) {
  __shared__ ScatterSmem<kScatterBlock, kScatterItems> sm;
  scatter_body<kScatterBlock, kScatterItems>(sm, keys, n, hist, fill, list);
}

// Both steps in one cooperative launch: every block counts its share of the
// pairs, the grid synchronises (the histogram is complete), then every block
// places its tiles.  The count's shared memory is reused by the scatter.
constexpr int kFusedItems = 16;
using FusedSmem = ScatterSmem<kCountBlock, kFusedItems>;
__global__ void __launch_bounds__(kCountBlock) order_pairs(const uint8_t* seq, int packed, const int64_t* p_off,
                                                            const int32_t* p_len, const int64_t* t_off,
                                                            const int32_t* t_len, int64_t n,
                                                            int32_t* max_len_sum, uint16_t* keys,
                                                            int32_t* hist, int32_t* fill, int64_t* list) {
  extern __shared__ __align__(16) uint8_t smem[];
  count_body(smem, seq, packed, p_off, p_len, t_off, t_len, n, max_len_sum, keys, hist);
  cooperative_groups::this_grid().sync();
  __syncthreads();
  scatter_body<kCountBlock, kFusedItems>(*reinterpret_cast<FusedSmem*>(smem), keys, n, hist, fill, list);
}

static cudaError_t allow_count_smem() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(order_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)order_count_smem());
  if (e == cudaSuccess) done = true;
  return e;
}

size_t order_count_smem() {
  return std::max((size_t)128 * kCountBlock * 4 + (size_t)kOrderBins * 4, sizeof(FusedSmem));
}

cudaError_t launch_order_count(const uint8_t* seq, int packed, const int64_t* p_off, const int32_t* p_len,
                               const int64_t* t_off, const int32_t* t_len, int64_t n, int num_sms,
                               int32_t* max_len_sum, uint16_t* keys, int32_t* hist, cudaStream_t st) {
  cudaError_t e = allow_count_smem();
  if (e != cudaSuccess) return e;
  const int64_t want = (n + kCountBlock - 1) / kCountBlock;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * 3));
  order_count<<<blocks, kCountBlock, order_count_smem(), st>>>(seq, packed, p_off, p_len, t_off, t_len, n,
                                                               max_len_sum, keys, hist);
  return cudaGetLastError();
}

cudaError_t launch_order_scatter(const uint16_t* keys, int64_t n, const int32_t* hist, int32_t* fill,
                                 int64_t* list, int num_sms, cudaStream_t st) {
  const int64_t tiles = (n + kScatterTile - 1) / kScatterTile;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)num_sms * 8));
  order_scatter<<<blocks, kScatterBlock, 0, st>>>(keys, n, hist, fill, list);
  return cudaGetLastError();
}

// Loads the ordering kernels (CUDA loads a kernel at its first launch
// otherwise; see preload_kernels in wfa_capi.cu).
cudaError_t preload_order_kernels() {
  cudaFuncAttributes a;
  for (const void* f : {(const void*)order_count, (const void*)order_scatter, (const void*)order_pairs}) {
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_order(const uint8_t* seq, int packed, const int64_t* p_off, const int32_t* p_len,
                         const int64_t* t_off, const int32_t* t_len, int64_t n, int num_sms, int32_t* max_len_sum,
                         uint16_t* keys, int32_t* hist, int32_t* fill, int64_t* list, cudaStream_t st,
                         int* launches) {
  cudaError_t e = allow_count_smem();
  if (e != cudaSuccess) return e;
  static int coop = -1, per_sm = 0;
  if (coop < 0) {
    int dev = 0, attr = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&attr, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && attr &&
        cudaFuncSetAttribute(order_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)order_count_smem()) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, order_pairs, kCountBlock, order_count_smem()) ==
            cudaSuccess &&
        per_sm > 0) {
      coop = 1;
    } else {
      cudaGetLastError();
      coop = 0;
    }
  }
  const int64_t want = (n + kCountBlock - 1) / kCountBlock;
  if (coop) {
    // Every block of a cooperative launch is resident at once.
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * std::min(per_sm, 3)));
    void* args[] = {(void*)&seq, (void*)&packed, (void*)&p_off, (void*)&p_len, (void*)&t_off, (void*)&t_len,
                    (void*)&n, (void*)&max_len_sum, (void*)&keys, (void*)&hist, (void*)&fill, (void*)&list};
    e = cudaLaunchCooperativeKernel((const void*)order_pairs, dim3(blocks), dim3(kCountBlock), args,
                                    order_count_smem(), st);
    if (e == cudaSuccess) {
      *launches = 1;
      return cudaSuccess;
    }
    cudaGetLastError();
  }
  e = launch_order_count(seq, packed, p_off, p_len, t_off, t_len, n, num_sms, max_len_sum, keys, hist, st);
  if (e != cudaSuccess) return e;
  *launches = 2;
  return launch_order_scatter(keys, n, hist, fill, list, num_sms, st);
}

}  // namespace wfab
