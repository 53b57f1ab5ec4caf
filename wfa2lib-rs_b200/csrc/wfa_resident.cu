// wfa_resident.cu -- the resident serving kernel: a persistent kernel that
// aligns single requests as the host publishes them.
//
// The host appends requests to a ring in mapped (zero-copy) pinned memory --
// a descriptor (lengths) and the pair's bytes per slot -- and publishes the
// count in `tail`.  One warp of the kernel (warp 0 of block 0, the doorbell)
// polls `tail` across the bus and mirrors it into device memory; every other
// lane group takes a ticket from a device counter and serves that request
// once the mirrored tail passes it: it stages the bytes, aligns them end to
// end with the
// same per-pair aligner as the batch kernels, and writes the result record
// and CIGAR into mapped memory followed by the slot's completion mark.  So
// requests join while the kernel runs, and nothing is copied per request by
// the host but the submitted bytes.
//
// Every wait is bounded: the doorbell ends the kernel after `idle_polls`
// polls without a new request (or when the host sets `stop`), the lane
// groups then drain what was published and return; a group that polls
// `group_polls` times without work or stop counts itself in `gave_up` and
// returns.  The host relaunches the kernel when requests arrive after it
// ended.
#include <cuda_runtime.h>

#include <mutex>

#include "wfa_align.cuh"
#include "wfa_kernels.h"
#include "wfa_resident.h"

namespace wfab {

WFA_D unsigned long long ld_volatile(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
WFA_D int32_t ld_volatile(const int32_t* p) { return *reinterpret_cast<const volatile int32_t*>(p); }

// The doorbell: mirrors the host's tail into device memory until the host
// stops the stream or no request arrives for R.idle_polls polls.
WFA_D void doorbell(const ResidentArgs& R) {
  unsigned long long seen = ld_volatile(R.dtail);
  int64_t idle = 0;
  for (;;) {
    const unsigned long long t = ld_volatile(&R.ctl->tail);
    if (t != seen) {
      seen = t;
      __threadfence_system();  // the requests below t are read after this
      *reinterpret_cast<volatile unsigned long long*>(R.dtail) = t;
      idle = 0;
    }
    if (ld_volatile(&R.ctl->stop)) {
      // The host published its last requests before setting stop.
      const unsigned long long t2 = ld_volatile(&R.ctl->tail);
      __threadfence_system();
      *reinterpret_cast<volatile unsigned long long*>(R.dtail) = t2;
      __threadfence();
      *reinterpret_cast<volatile int32_t*>(R.dstop) = 1;
      return;
    }
    if (++idle > R.idle_polls) {
      __threadfence();
      *reinterpret_cast<volatile int32_t*>(R.dstop) = 2;
      atomicAdd(&R.ctl->idle_exits, 1);
      return;
    }
    __nanosleep(400);
  }
}

// The next request for a lane group: lane 0 takes a ticket (one atomic add
// on the device counter) and waits until the doorbell has seen that many
// requests published; -1 when the stream stopped or went idle below the
// ticket (every ticket below the final tail is served before its group
// returns, so a relaunch starts at that tail), or when the group polled
// R.group_polls times (counted in gave_up; the host then fails the stream).
template <int LW>
WFA_D int64_t claim(const ResidentArgs& R, int lane) {
  long long slot = -1;
  if (lane == 0) {
    const unsigned long long ticket = atomicAdd(R.head, 1ull);
    int64_t polls = 0;
    unsigned ns = 64;
    for (;;) {
      if (ticket < ld_volatile(R.dtail)) {
        slot = (long long)ticket;
        break;
      }
      if (ld_volatile(R.dstop)) {
        // The doorbell stored the final tail before stop: one more look.
        if (ticket < ld_volatile(R.dtail)) continue;
        break;
      }
      if (++polls > R.group_polls) {
        atomicAdd(&R.ctl->gave_up, 1);
        break;
      }
      __nanosleep(ns);
      ns = ns < 4096 ? ns * 2 : ns;
    }
  }
  return (int64_t)__shfl_sync(Lanes<LW>::mask(), slot, 0, LW);
}

template <int CLS, int LW>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4) resident_kernel(const AlignParams P, const ResidentArgs R) {
  extern __shared__ __align__(16) uint8_t smem[];
  constexpr int kGroups = kWarpsPerBlock * 32 / LW;
  using G = Lanes<LW>;
  if (blockIdx.x == 0 && threadIdx.x < 32) {
    if (threadIdx.x == 0) doorbell(R);
    return;
  }
  const int gib = threadIdx.x / LW;
  const int lane = G::lane();
  const int64_t ggroup = (int64_t)blockIdx.x * kGroups + gib;
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const int slots = cell_slots(P, NC);
  const SmemLayout L = smem_layout(P.desc_depth ? P.desc_depth : P.scope, NC, slots, P.ring_smem ? P.wmax : 0,
                                   P.seq_smem_words, kGroups);
  Workspace ws;
  ws.ring = reinterpret_cast<WfD*>(smem + L.desc_off + (size_t)gib * L.desc_bytes);
  int32_t* slice = P.scratch + ggroup * P.warp_words;
  const int64_t ring_words = slice_ring_words(P, NC);
  ws.ringv = P.ring_smem ? reinterpret_cast<int32_t*>(smem + L.ring_off + (size_t)gib * L.ring_bytes) : slice;
  ws.ringg = P.ring_smem && P.ring_slots > 0 && P.wspill > 0 ? slice : nullptr;
  ws.hist = reinterpret_cast<int4*>(slice + ring_words);
  ws.harena = slice + ring_words + (int64_t)P.hist_scores * 4;
  ws.dom = nullptr;
  ws.bt = nullptr;
  ws.btinit = nullptr;
  ws.btmark = nullptr;
  // After the ring and history (16-byte aligned): the request's bytes and
  // its CIGAR.
  uint8_t* stage = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(ws.harena + P.hist_words) + 15) & ~(uintptr_t)15);
  uint8_t* cg_stage = stage + R.seq_stride;
  for (;;) {
    const int64_t slot = claim<LW>(R, lane);
    if (slot < 0) break;
    const int64_t i = slot % R.cap;
    // The slot was written by the host after any earlier read of its cache
    // lines (a neighbouring slot's descriptor, the slot's previous request):
    // read it with loads that fetch again (ld.cv) rather than from a cache.
    __threadfence_system();
    const int2 q = __ldcv(reinterpret_cast<const int2*>(R.reqs) + i);
    const int n = q.x, m = q.y;
    // Stage the request's bytes (pattern then text) in device memory: the
    // aligner reads them many times.
    const int4* src = reinterpret_cast<const int4*>(R.arena + i * R.seq_stride);
    int4* dst = reinterpret_cast<int4*>(stage);
    for (int w = lane; w < (n + m + 15) / 16; w += LW) dst[w] = __ldcv(src + w);
    G::sync();
    SeqAscii sp{stage, n};
    SeqAscii st{stage + n, m};
    PairAligner<CLS, SeqAscii, false, 1, LW, false> A(P);
    A.ws = ws;
    A.lane = lane;
    A.pat = sp;
    A.txt = st;
    A.n = n;
    A.m = m;
    A.scope = P.scope;
    A.wmax = P.wmax;
    A.compact = P.ring_slots > 0;
    A.modular = P.compute_alignment == 0;
    A.pgb = false;
    A.cap = A.modular ? INT_MAX : imax(A.dims_num(1000, 1000), A.dims_num(n, m));
    A.endsfree = false;
    A.hkind = WFA_HEURISTIC_NONE; A.hp0 = A.hp1 = A.hp2 = 0;
    A.hist_nc = 1;
    A.pcoff = 0;
    A.mbase = nullptr;
    A.keep_null_slots = false;
    A.comp_end = CM;
    A.p0 = A.pf = A.t0 = A.tf = 0;
    A.cg = A.modular ? nullptr : cg_stage;
    A.cg_cap = A.modular ? 0 : 2 * ((int64_t)n + m) + 1;
    const int32_t score = A.align();
    const bool has = A.status != kStatusRetry && A.cg_end > A.cg_begin && !A.modular;
    const int64_t len = has ? A.cg_end - A.cg_begin : 0;
    uint8_t* cdst = R.cigars + i * R.cig_stride;
    for (int64_t j = lane; j < len; j += LW) cdst[j] = A.cg[A.cg_begin + j];
    if (lane == 0) {
      wfa_result_t r;
      r.score = A.status == kStatusRetry ? 0 : score;
      r.status = A.status;
      r.cigar_begin = 0;
      r.cigar_length = (int32_t)len;
      r.cigar_score = A.cg_score;
      r.end_v = A.cg_ev;
      r.end_h = A.cg_eh;
      r.end_score = A.end_score;
      r.end_k = A.end_k;
      r.end_offset = A.end_off;
      R.results[i] = r;
    }
    // Every lane's writes reach the host before the completion mark.
    __threadfence_system();
    G::sync();
    if (lane == 0) {
      __threadfence_system();
      *reinterpret_cast<volatile uint32_t*>(R.done + i) = (uint32_t)(slot / R.cap) + 1u;
    }
    G::sync();
  }
}

template <int CLS, int LW>
static cudaError_t launch_res_t(const AlignParams& P, const ResidentArgs& R, int blocks, size_t smem,
                                cudaStream_t st) {
  auto k = resident_kernel<CLS, LW>;
  static size_t configured = 0;
  static bool carveout = false;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lock(mu);
    // The SMs that host the resident kernel keep its shared-memory
    // configuration while it runs: ask for the largest, so that other
    // kernels' blocks (larger shared-memory needs) fit beside it instead of
    // waiting for it to end.
    if (!carveout) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return e;
      carveout = true;
    }
    if (smem > configured) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      configured = smem;
    }
  }
  k<<<blocks, kWarpsPerBlock * 32, smem, st>>>(P, R);
  return cudaGetLastError();
}

template <int CLS, int LW>
static int occ_res_t(size_t smem) {
  int nb = 0;
  cudaFuncAttributes fa;  // loads the kernel if it is not yet
  if (cudaFuncGetAttributes(&fa, resident_kernel<CLS, LW>) != cudaSuccess) cudaGetLastError();
  if (cudaFuncSetAttribute(resident_kernel<CLS, LW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, resident_kernel<CLS, LW>, kWarpsPerBlock * 32, smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return nb < 1 ? 1 : nb;
}

cudaError_t launch_resident(const AlignParams& P, const ResidentArgs& R, int cls, int lanes, int blocks,
                            size_t smem, cudaStream_t st) {
  const bool w8 = lanes == 8;
  switch (cls) {
    case kEditClass: return w8 ? launch_res_t<kEditClass, 8>(P, R, blocks, smem, st)
                               : launch_res_t<kEditClass, 32>(P, R, blocks, smem, st);
    case kLinearClass: return w8 ? launch_res_t<kLinearClass, 8>(P, R, blocks, smem, st)
                                 : launch_res_t<kLinearClass, 32>(P, R, blocks, smem, st);
    case kAffineClass: return w8 ? launch_res_t<kAffineClass, 8>(P, R, blocks, smem, st)
                                 : launch_res_t<kAffineClass, 32>(P, R, blocks, smem, st);
    default: return w8 ? launch_res_t<kAffine2pClass, 8>(P, R, blocks, smem, st)
                       : launch_res_t<kAffine2pClass, 32>(P, R, blocks, smem, st);
  }
}

int occupancy_resident(int cls, int lanes, size_t smem) {
  const bool w8 = lanes == 8;
  switch (cls) {
    case kEditClass: return w8 ? occ_res_t<kEditClass, 8>(smem) : occ_res_t<kEditClass, 32>(smem);
    case kLinearClass: return w8 ? occ_res_t<kLinearClass, 8>(smem) : occ_res_t<kLinearClass, 32>(smem);
    case kAffineClass: return w8 ? occ_res_t<kAffineClass, 8>(smem) : occ_res_t<kAffineClass, 32>(smem);
    default: return w8 ? occ_res_t<kAffine2pClass, 8>(smem) : occ_res_t<kAffine2pClass, 32>(smem);
  }
}

}  // namespace wfab
