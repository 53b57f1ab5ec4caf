// wfa_capi.cu -- host side of the C ABI (include/wfa_b200.h).
//
// A handle mirrors one reference WavefrontAligner (src/aligner.rs:146): its
// builder state, the last alignment's status and CIGAR, and the device
// resources it reuses across calls (input/output buffers, per-warp scratch,
// a stream).  Alignments always run on the GPU: there is no CPU path, and a
// configuration this build cannot run on the device is refused with
// WFA_ERR_UNSUPPORTED.
#include <cuda_runtime.h>

#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wfa_common.h"
#include "wfa_kernels.h"
#include "wfa_noalloc.h"
#include "wfa_params.h"
#include "wfa_resident.h"

using namespace wfab;

namespace {

// A device buffer that grows on demand.  Growing uses stream-ordered
// allocation on the handle's stream: cudaFree would wait for every kernel on
// the device (other handles' and other threads' included), while the
// stream-ordered free waits only for this stream, whose earlier work the
// callers have already synchronised.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaStream_t st = nullptr;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)256);
    cudaError_t e = cudaMallocAsync(&p, want, st);
    // Usable from the handle's other streams once the allocation is done.
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

struct ScratchCfg {
  int32_t wmax;
  int32_t ring_slots = 0;  // compact ring slots (0: one per score and component)
  int32_t bt_cap = 0, bt_init_cap = 0;  // med/low backtrace buffer (blocks, initial positions)
  int32_t hist_scores;
  int64_t hist_words;
  int64_t dom_words = 0;  // Corrected-mode dominance array per warp
};

}  // namespace

struct wfa_aligner {
  int device = 0;
  AlignParams pen{};  // penalties and scope (set_penalties)
  int memory_mode = WFA_MEMORY_HIGH;
  uint64_t max_memory_compact = 256ull << 20;
  int compat = WFA_COMPAT_C;
  int scope = WFA_SCOPE_SCORE;  // the reference's default (src/aligner.rs:433)
  int span = WFA_SPAN_END2END;
  int extension = 0;
  int32_t p0 = 0, pf = 0, t0 = 0, tf = 0;
  int hkind = WFA_HEURISTIC_NONE;
  int32_t hp0 = 0, hp1 = 0, hp2 = 0;
  int32_t max_steps = INT32_MAX;
  // last plain alignment
  int status = WFA_STATUS_OK;
  std::vector<uint8_t> cigar;
  int32_t cigar_score = INT32_MIN, end_v = -1, end_h = -1;
  int32_t end_score = -1, end_k = kDiagNull, end_offset = kOffsetNull;
  int last_err = WFA_OK;
  std::string err_str;
  // device resources
  cudaStream_t stream = nullptr;    // compute (every kernel of the handle)
  cudaStream_t s_in = nullptr;      // host->device copies
  cudaStream_t s_out = nullptr;     // device->host copies
  cudaStream_t s_cig = nullptr;     // device->host copies of packed CIGARs (host-buffer batch)
  int num_sms = 148;
  DevBuf seq, poff, plen, toff, tlen, coff, results, cigars, dense, scratch, counters, pairlist;
  DevBuf chunkinfo;               // per-chunk counters and dense CIGAR ranges
  DevBuf order;                   // cost ordering: keys, histograms, pair lists
  DevBuf checks;                  // device-checks build: failed index checks
  int64_t* hinfo = nullptr;       // pinned host copy of the chunk info
  size_t hinfo_cap = 0;
  int64_t launches = 0;
  uint8_t* pinned = nullptr;  // host staging for the plain per-call form
  size_t pinned_cap = 0;
  int occ_key = -1;
  size_t occ_smem = 0;
  int occ_val = 1;
  int lanes_forced = 0;  // lanes per pair of the lean kernel (0: autotuned)
  int bi_lanes_forced = 0;  // lanes per pair of the BiWFA kernel (0: by length)
  int last_lanes = 0;    // lanes per pair of the last batch's first round
  int launch_lanes = 0;  // lanes per pair of the last launch
  int64_t last_slice_bytes = 0;  // one lane group's scratch slice in the last launch
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_kernel_ms = 0.0;
  int64_t last_reruns = 0;  // pair re-runs (larger scratch) of the last call
  // Events of the pipelined host-buffer batch, created once and reused:
  // creating and destroying events waits for work running on the device
  // (other handles' kernels included).
  std::vector<cudaEvent_t> evpool;
  std::vector<cudaEvent_t> evtime;  // timing events around each chunk's alignment kernel
  // Asynchronous host-buffer batches (wfa_batch_submit): one worker thread,
  // started by the first submit, runs them in submission order.
  struct Job {
    int64_t ticket;
    wfa_batch_t batch;
    wfa_result_t* results;
    uint8_t* cigars;
  };
  std::thread async_worker;
  std::mutex async_mu;
  std::condition_variable async_cv;
  std::deque<Job> async_jobs;
  std::map<int64_t, int> async_done;  // ticket -> return code
  int64_t async_next = 0;
  bool async_stop = false;
};

// At least `count` pooled events in h->evpool.
// Pinned host words for the per-chunk info of the host-buffer batch.
static cudaError_t host_info(wfa_aligner_t* h, size_t words) {
  if (h->hinfo_cap >= words) return cudaSuccess;
  if (h->hinfo) cudaFreeHost(h->hinfo);
  h->hinfo = nullptr;
  h->hinfo_cap = 0;
  void* p = nullptr;
  cudaError_t e = cudaHostAlloc(&p, std::max<size_t>(words, 64) * 8, cudaHostAllocDefault);
  if (e != cudaSuccess) return e;
  h->hinfo = static_cast<int64_t*>(p);
  h->hinfo_cap = std::max<size_t>(words, 64);
  return cudaSuccess;
}

// What the host-buffer batch needs to know of a chunk of pairs before it is
// copied in: the byte range of the sequence buffer it reads (16-byte
// aligned), its longest pair (n + m) and its CIGAR slot bytes.
struct ChunkInfo {
  int64_t lo = INT64_MAX, hi = 0;
  int32_t max_len_sum = 0;
  int32_t max_seq = 0;  // longest single sequence
  int64_t slots = 0;
};
static void scan_chunks(const wfa_batch_t* b, int64_t n, const std::vector<int64_t>& bnd, bool packed,
                        bool aln, std::vector<ChunkInfo>& out) {
  const int64_t nchunks = (int64_t)out.size();
  const int64_t unit = packed ? 4 : 1;  // bytes per offset unit
  // One pass over [i0, i1), accumulated per chunk into `acc`.
  auto pass = [&](int64_t i0, int64_t i1, std::vector<ChunkInfo>& acc) {
    int64_t ci = std::upper_bound(bnd.begin(), bnd.end(), i0) - bnd.begin() - 1;
    for (int64_t i = i0; i < i1; ++ci) {
      const int64_t e = std::min(i1, bnd[(size_t)ci + 1]);
      ChunkInfo& c = acc[(size_t)ci];
      int64_t lo = c.lo, hi = c.hi, slots = c.slots;
      int32_t mx = c.max_len_sum, ms = c.max_seq;
      for (; i < e; ++i) {
        const int64_t pl = b->p_len[i], tl = b->t_len[i], po = b->p_off[i], to = b->t_off[i];
        const int64_t pe = packed ? (po + (pl + 15) / 16) * 4 : po + pl;
        const int64_t te = packed ? (to + (tl + 15) / 16) * 4 : to + tl;
        lo = std::min(lo, std::min(po, to) * unit);
        hi = std::max(hi, std::max(pe, te));
        mx = std::max<int32_t>(mx, (int32_t)(pl + tl));
        ms = std::max<int32_t>(ms, (int32_t)std::max(pl, tl));
        slots += 2 * (pl + tl) + 1;
      }
      c.lo = lo; c.hi = hi; c.slots = slots; c.max_len_sum = mx; c.max_seq = ms;
    }
  };
  const int64_t kPerThread = 131072;
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(8, n / kPerThread));
  std::vector<std::vector<ChunkInfo>> part((size_t)nt, std::vector<ChunkInfo>((size_t)nchunks));
  if (nt == 1) {
    pass(0, n, part[0]);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
      th.emplace_back(pass, n * t / nt, n * (t + 1) / nt, std::ref(part[(size_t)t]));
    for (auto& x : th) x.join();
  }
  for (int64_t ci = 0; ci < nchunks; ++ci) {
    ChunkInfo c;
    for (int t = 0; t < nt; ++t) {
      const ChunkInfo& p = part[(size_t)t][(size_t)ci];
      c.lo = std::min(c.lo, p.lo);
      c.hi = std::max(c.hi, p.hi);
      c.max_len_sum = std::max(c.max_len_sum, p.max_len_sum);
      c.max_seq = std::max(c.max_seq, p.max_seq);
      c.slots += p.slots;
    }
    c.lo = c.lo == INT64_MAX ? 0 : (c.lo & ~(int64_t)15);
    c.hi = std::min<int64_t>(b->seq_bytes, (c.hi + 15) & ~(int64_t)15);
    if (!aln) c.slots = 0;
    out[(size_t)ci] = c;
  }
}

static cudaError_t event_pool(wfa_aligner_t* h, size_t count) {
  while (h->evpool.size() < count) {
    cudaEvent_t e = nullptr;
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) return r;
    h->evpool.push_back(e);
  }
  return cudaSuccess;
}

// At least `count` pooled events that record time.
static cudaError_t timing_events(wfa_aligner_t* h, size_t count) {
  while (h->evtime.size() < count) {
    cudaEvent_t e = nullptr;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    h->evtime.push_back(e);
  }
  return cudaSuccess;
}

static int fail(wfa_aligner_t* h, int code, const char* what, cudaError_t e = cudaSuccess) {
  if (h) {
    h->last_err = code;
    h->err_str = what;
    if (e != cudaSuccess) {
      h->err_str += ": ";
      h->err_str += cudaGetErrorString(e);
    }
  }
  return code;
}

#define CUDA_TRY(h, expr, what)                                             \
  do {                                                                     \
    cudaError_t _e = (expr);                                               \
    if (_e != cudaSuccess) {                                               \
      return fail(h, _e == cudaErrorMemoryAllocation ? WFA_ERR_OOM : WFA_ERR_CUDA, what, _e); \
    }                                                                      \
  } while (0)

// ---------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------
__global__ void collect_retries(const wfa_result_t* res, const int64_t* list, int64_t n,
                                int64_t* out, int32_t* count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t pair = list ? list[i] : i;
  if (res[pair].status == kStatusRetry) {
    int32_t slot = atomicAdd(count, 1);
    out[slot] = pair;
  }
}

// Copies every pair's CIGAR from its slot to dense[dst_off[i]..] (one warp
// per pair, coalesced byte copies) and makes that its cigar_begin.
__global__ void compact_cigars(wfa_result_t* res, const int64_t* slot_off,
                               const uint8_t* slots, const int64_t* dst_off, uint8_t* dense,
                               int64_t n) {
  int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= n || res[w].status == kStatusRetry) return;  // retried pairs are copied later
  int32_t len = res[w].cigar_length;
  const uint8_t* src = slots + slot_off[w] + res[w].cigar_begin;
  uint8_t* dst = dense + dst_off[w];
  for (int32_t i = lane; i < len; i += 32) dst[i] = src[i];
  __syncwarp();
  if (lane == 0) res[w].cigar_begin = (int32_t)dst_off[w];  // now an offset into the dense bytes
}

// Exclusive prefix sums of a chunk's per-pair values, in three short
// launches (tile sums, a one-block scan of the tile sums, the tiles' own
// scans): MODE 0 the CIGAR slot sizes 2 (n + m) + 1 from the lengths, MODE 1
// the CIGAR lengths of the results (0 for pairs to be re-run).
constexpr int kScanBlock = 256, kScanItems = 8, kScanTile = kScanBlock * kScanItems;
template <int MODE>
__device__ __forceinline__ long long scan_value(const int32_t* pl, const int32_t* tl,
                                                const wfa_result_t* res, int64_t i) {
  if (MODE == 0) return 2ll * ((long long)pl[i] + tl[i]) + 1;
  return res[i].status == kStatusRetry ? 0 : res[i].cigar_length;
}
template <int MODE, bool APPLY>
__global__ void __launch_bounds__(kScanBlock)
    scan_tiles(const int32_t* pl, const int32_t* tl, const wfa_result_t* res, int64_t n,
               long long* tile, int64_t* out) {
  using Scan = cub::BlockScan<long long, kScanBlock>;
  __shared__ typename Scan::TempStorage tmp;
  const int64_t i0 = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  long long v[kScanItems], sum = 0;
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = i0 + j < n ? scan_value<MODE>(pl, tl, res, i0 + j) : 0;
    sum += v[j];
  }
  long long excl, total;
  Scan(tmp).ExclusiveSum(sum, excl, total);
  if (!APPLY) {
    if (threadIdx.x == 0) tile[blockIdx.x] = total;
    return;
  }
  long long run = tile[blockIdx.x] + excl;
  for (int j = 0; j < kScanItems; ++j) {
    if (i0 + j < n) out[i0 + j] = run;
    run += v[j];
  }
}
// The tile sums in place become tile offsets from the chunk's base: `base0`,
// or *base (then advanced past the chunk).  range = [begin, end).
__global__ void __launch_bounds__(1024)
    scan_tile_offsets(long long* tile, int64_t ntiles, int64_t base0, int64_t* base, int64_t* range) {
  using Scan = cub::BlockScan<long long, 1024>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = base ? *base : base0;
  __syncthreads();
  const long long begin = carry;
  for (int64_t t0 = 0; t0 < ntiles; t0 += 1024) {
    const int64_t t = t0 + threadIdx.x;
    const long long v = t < ntiles ? tile[t] : 0;
    long long excl, total;
    Scan(tmp).ExclusiveSum(v, excl, total);
    if (t < ntiles) tile[t] = carry + excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (base) *base = carry;
    if (range) { range[0] = begin; range[1] = carry; }
  }
}
template <int MODE>
static cudaError_t chunk_scan(const int32_t* pl, const int32_t* tl, const wfa_result_t* res, int64_t n,
                              int64_t base0, int64_t* base, int64_t* out, int64_t* range, long long* tile,
                              cudaStream_t st) {
  const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
  if (ntiles > 0) scan_tiles<MODE, false><<<(unsigned)ntiles, kScanBlock, 0, st>>>(pl, tl, res, n, tile, out);
  scan_tile_offsets<<<1, 1024, 0, st>>>(tile, ntiles, base0, base, range);
  if (ntiles > 0) scan_tiles<MODE, true><<<(unsigned)ntiles, kScanBlock, 0, st>>>(pl, tl, res, n, tile, out);
  return cudaGetLastError();
}

// out[0]: the longest n + m of a batch; out[1]: its longest sequence.
__global__ void max_lengths(const int32_t* pl, const int32_t* tl, int64_t n, int32_t* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t v = 0, w = 0;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v = max(v, pl[i] + tl[i]);
    w = max(w, max(pl[i], tl[i]));
  }
  v = __reduce_max_sync(0xffffffffu, v);
  w = __reduce_max_sync(0xffffffffu, w);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, v);
    atomicMax(out + 1, w);
  }
}

// ---------------------------------------------------------------------------
// Configuration checks
// ---------------------------------------------------------------------------
static int check_supported(wfa_aligner_t* h, bool biwfa) {
  if (h->pen.scope > 1024) return fail(h, WFA_ERR_UNSUPPORTED, "max_score_scope above 1024");
  return WFA_OK;
}

static void fill_params(const wfa_aligner_t* h, const wfa_batch_t* b, AlignParams& P) {
  P = h->pen;
  P.span = b->span == WFA_SPAN_BIWFA ? WFA_SPAN_END2END : b->span;
  P.extension = b->span == WFA_SPAN_ENDSFREE ? h->extension : 0;
  P.p0 = h->p0; P.pf = h->pf; P.t0 = h->t0; P.tf = h->tf;
  P.hkind = h->hkind; P.hp0 = h->hp0; P.hp1 = h->hp1; P.hp2 = h->hp2;
  P.compute_alignment = h->scope == WFA_SCOPE_ALIGNMENT;
#ifdef WFA_DEVICE_CHECKS
  P.check_count = h->checks.as<int32_t>();
#else
  P.check_count = nullptr;
#endif
  // Med/low with an alignment: the piggyback backtrace (BiWFA ignores the mode).
  P.piggyback = P.compute_alignment && h->memory_mode != WFA_MEMORY_HIGH && b->span != WFA_SPAN_BIWFA
                    ? (h->memory_mode == WFA_MEMORY_LOW ? 2 : 1)
                    : 0;
  P.bt_limit = (int64_t)std::min<uint64_t>(h->max_memory_compact, (uint64_t)INT64_MAX);
  P.bt_probe = kProbeIntervalCompact;
  P.compat = h->compat;
  P.max_steps = h->max_steps;
  P.format = b->format;
  P.seq = static_cast<const uint8_t*>(b->seq);
  P.seq_bytes = b->seq_bytes;
  P.p_off = b->p_off; P.p_len = b->p_len; P.t_off = b->t_off; P.t_len = b->t_len;
  P.cigar_off = b->cigar_off;
  P.num_pairs = b->num_pairs;
  P.pair_list = nullptr;
}

// Scratch configuration of one launch over pairs whose longest has
// n + m = max_len_sum.  The unidirectional kernel keeps the compact ring
// (compact_ring_slots): for pairs up to kLongPair its cells sit in shared
// memory, rows wider than the shared-memory slot going to a spill ring in
// the lane group's scratch slice as wide as any wavefront of the launch can
// be, so only an M history that outgrows its slice makes a pair re-run;
// sequences short enough are staged in shared memory too.  Longer pairs keep
// the whole ring in the scratch slice.  Pairs that outgrow a configuration
// are re-run with a larger one (next_round).
static constexpr int kSeqSmemWords = 64;
static constexpr size_t kScratchBudget = (size_t)6 << 30;

// Scratch may grow to half of the device memory that is free (counting the
// scratch buffer already held), at least kScratchBudget and at most 64 GiB.
static size_t scratch_budget(wfa_aligner_t* h) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return kScratchBudget;
  }
  return std::max(kScratchBudget, std::min((size_t)64 << 30, (fr + h->scratch.cap) / 2));
}

struct Round {
  ScratchCfg cfg;
  bool ring_smem;
  int lanes;         // lanes per pair (4, 8, 16 or 32)
  int32_t wspill;    // spill ring width (0: none)
  int32_t seq_words; // words per sequence staged in shared memory
};

// Long pairs (n + m above kLongPair) start with the ring in the scratch
// slice and an M history sized from their lengths: a re-run after an overflow
// late in a long alignment repeats most of its work.
static constexpr int32_t kLongPair = 2048;

// The widest wavefront storage a pair can need: computed diagonals are
// clamped to [-(n + scope + 1), m + scope + 1] (src/aligner.rs:915-924), and a
// score with begin-free seeds (k = score / -match <= max(n, m)) covers
// [-k, k] as well (:3426-3452).  Searches that run on past the sequence ends
// (Corrected ends-free, whole-length free ends) reach these bounds.
static int32_t max_width(const AlignParams& P, int32_t max_len_sum) {
  return 2 * (max_len_sum + P.scope) + 5;
}

// Shared-memory slot width of the compact ring per lane-group width: narrow
// groups keep many pairs in flight per SM, each with a narrower slot (rows
// above it spill).
static int32_t smem_slot_width(int lanes) { return lanes == 4 ? 16 : lanes == 8 ? 32 : 64; }

static Round first_round(const AlignParams& P, int nc, int32_t max_len_sum, int lanes = 32,
                         bool spill = true, int32_t max_seq = 0) {
  Round r;
  const int cls = metric_class(P.metric);
  const bool longp = max_len_sum > kLongPair;
  r.lanes = lanes;
  r.cfg.wmax = std::max(8, std::min(max_width(P, max_len_sum), 8192));
  r.cfg.ring_slots = compact_ring_slots(P, cls);
  // The piggyback backtrace keeps every component's history.
  const int hnc = P.piggyback ? nc : 1;
  r.cfg.hist_scores = P.compute_alignment ? hnc * (longp ? max_len_sum + 3 : 1024) : 0;
  r.cfg.hist_words = P.compute_alignment
                         ? hnc * (int64_t)std::max(32768, (longp ? 64 : 16) * (max_len_sum + 3))
                         : 0;
  r.ring_smem = !longp;
  r.wspill = 0;
  if (P.piggyback) {
    // Med/low keep no history: the ring (offsets, pcigars and block indices,
    // as wide as any wavefront of the launch) and a backtrace buffer sized
    // from the lengths, grown when a pair outgrows it.
    r.ring_smem = false;
    r.cfg.hist_scores = 0;
    r.cfg.hist_words = 0;
    r.cfg.bt_cap = std::max(16384, 16 * (max_len_sum + 3));
    r.cfg.bt_init_cap = max_len_sum + 8;
  }
  if (r.ring_smem) {
    const int32_t wsm = smem_slot_width(lanes);
    if (spill && r.cfg.wmax > wsm) r.wspill = r.cfg.wmax;
    r.cfg.wmax = std::min(r.cfg.wmax, wsm);
  }
  // The longest sequence of the launch (max_seq, else at most max_len_sum).
  const bool packed = P.format == WFA_SEQ_PACKED2;
  const int32_t ms = max_seq > 0 ? max_seq : max_len_sum;
  r.seq_words = std::min(kSeqSmemWords, packed ? (ms + 15) / 16 : (ms + 3) / 4 + 1);
  r.seq_words = (r.seq_words + 1) & ~1;
  // Corrected ends-free with begin-free seeds prunes dominated cells against
  // a per-diagonal array over [-(n + scope + 2), m + scope + 2] per component.
  const bool dom = P.compat == WFA_COMPAT_CORRECTED && P.match < 0 && P.span == WFA_SPAN_ENDSFREE &&
                   !P.extension && std::max(P.p0, P.t0) > 0;
  r.cfg.dom_words = dom ? (int64_t)nc * ((int64_t)max_len_sum + 2 * P.scope + 5) : 0;
  return r;
}

static void next_round(Round& r, const AlignParams& P, int32_t max_len_sum) {
  const int32_t full = std::max(8, std::min(max_width(P, max_len_sum), 8192));
  if (r.ring_smem && r.wspill == 0) {
    r.ring_smem = false;  // retries use the scratch ring at full width
    r.cfg.wmax = full;
  } else if (!r.ring_smem) {
    r.cfg.wmax = std::min(max_width(P, max_len_sum), std::max(r.cfg.wmax, 1) * 4);
  }
  // (with a spill ring, every row already fits: only the history grows)
  if (P.compute_alignment) {
    r.cfg.hist_scores *= 4;
    r.cfg.hist_words *= 4;
  }
  if (P.piggyback) r.cfg.bt_cap = (int32_t)std::min<int64_t>((int64_t)r.cfg.bt_cap * 4, INT32_MAX / 2);
}

// Fills the launch fields of P for round r and returns the per-block shared
// memory and the words of one lane group's scratch slice.
static SmemLayout round_layout(AlignParams& P, const Round& r, int nc, int64_t* group_words) {
  P.seq_smem_words = r.seq_words;
  P.ring_smem = r.ring_smem ? 1 : 0;
  P.wmax = r.cfg.wmax;
  P.ring_slots = r.cfg.ring_slots;
  P.desc_depth = r.cfg.ring_slots ? compact_desc_depth(P, metric_class(P.metric)) : 0;
  P.wspill = r.wspill;
  P.hist_scores = r.cfg.hist_scores;
  P.hist_words = r.cfg.hist_words;
  P.dom_words = r.cfg.dom_words;
  P.bt_cap = r.cfg.bt_cap;
  P.bt_init_cap = r.cfg.bt_init_cap;
  const int groups = kWarpsPerBlock * 32 / r.lanes;
  const SmemLayout L = smem_layout(P.desc_depth ? P.desc_depth : P.scope, nc, cell_slots(P, nc),
                                   r.ring_smem ? r.cfg.wmax : 0, r.seq_words, groups);
  int64_t w = slice_ring_words(P, nc) + (int64_t)r.cfg.hist_scores * 4 +
              ((r.cfg.hist_words + r.cfg.dom_words + 3) & ~(int64_t)3) + slice_bt_words(P);
  *group_words = std::max<int64_t>((w + 63) & ~(int64_t)63, 64);
  return L;
}

// Resident blocks per SM of the round's kernel (cached per handle).
static int round_occupancy(wfa_aligner_t* h, const AlignParams& P, int cls, int lanes, size_t smem) {
  const int key = ((cls * 4 + (P.format == WFA_SEQ_PACKED2) * 2 + (needs_general(P) ? 1 : 0)) << 6) | lanes;
  if (key != h->occ_key || smem != h->occ_smem) {
    h->occ_val = occupancy_blocks_per_sm(P, cls, lanes, smem);
    h->occ_key = key;
    h->occ_smem = smem;
  }
  return h->occ_val;
}

// Sizes the scratch for round r and launches the alignment kernel over
// `todo` pairs (`list`: their indices, or NULL for 0..todo-1).  No sync.
static int launch_round(wfa_aligner_t* h, AlignParams& P, const Round& r0, int64_t todo,
                        const int64_t* list, cudaStream_t st, unsigned long long* ctr = nullptr) {
  const int cls = metric_class(P.metric);
  const int nc = metric_components(P.metric);
  int64_t group_words = 0;
  // Narrow lane groups keep more rings in a block; a large score scope
  // (penalties with a match reward) may not fit them, then wider groups run.
  Round r = r0;
  SmemLayout L = round_layout(P, r, nc, &group_words);
  while (L.total > 200 * 1024 && r.lanes < 32) {
    r.lanes *= 2;
    L = round_layout(P, r, nc, &group_words);
  }
  h->launch_lanes = r.lanes;
  const size_t smem = L.total;
  if (smem > 200 * 1024) return fail(h, WFA_ERR_UNSUPPORTED, "wavefront ring too large");
  const int occ = round_occupancy(h, P, cls, r.lanes, smem);
  const int gpb = kWarpsPerBlock * 32 / r.lanes;  // lane groups per block
  int64_t max_groups = (int64_t)h->num_sms * occ * gpb;
  int64_t groups = std::max<int64_t>(std::min<int64_t>(max_groups, todo), 1);
  const size_t budget =
      (size_t)groups * group_words * 4 > kScratchBudget ? scratch_budget(h) : kScratchBudget;
  while (groups > gpb && (size_t)groups * group_words * 4 > budget) groups /= 2;
  int blocks = (int)((groups + gpb - 1) / gpb);
  size_t scratch_bytes = (size_t)blocks * gpb * group_words * 4;
  CUDA_TRY(h, h->scratch.ensure(scratch_bytes), "scratch");
  CUDA_TRY(h, h->counters.ensure(64), "counters");
  P.scratch = h->scratch.as<int32_t>();
  P.warp_words = group_words;
  h->last_slice_bytes = group_words * 4;
  P.work_counter = ctr ? ctr : h->counters.as<unsigned long long>();
  P.retry_count = reinterpret_cast<int32_t*>(P.work_counter + 1);
  P.pair_list = list;
  P.num_pairs = todo;
  CUDA_TRY(h, cudaMemsetAsync(P.work_counter, 0, 16, st), "memset");
  CUDA_TRY(h, cudaEventRecord(h->ev0, st), "event");
  CUDA_TRY(h, cudaGetLastError(), "an earlier CUDA call of this thread");
  CUDA_TRY(h, launch_unialign(P, cls, r.lanes, blocks, smem, st), "alignment kernel launch");
  CUDA_TRY(h, cudaEventRecord(h->ev1, st), "event");
  h->launches++;
  return WFA_OK;
}

// ---------------------------------------------------------------------------
// Lanes per pair of the lean kernel, autotuned per length bucket
// ---------------------------------------------------------------------------
// The first device batch of a (device, metric class, encoding, CIGAR or
// score, length bucket) times each candidate lane-group width on a sample of
// its pairs (the first kTuneSample of its cost order, twice each, the faster
// run counting) and keeps the fastest for the process; the general kernel
// always takes whole warps.  Results do not depend on the width: every width runs the same
// per-pair algorithm.
static constexpr int64_t kTuneSample = 1 << 20, kTuneMinPairs = 65536;

static int length_bucket(int32_t max_len_sum) {
  return max_len_sum <= 384 ? 0 : max_len_sum <= 1024 ? 1 : max_len_sum <= kLongPair ? 2 : 3;
}
static int default_lanes(const AlignParams& P, int bucket) {
  if (needs_general(P) || bucket == 3) return 32;
  return bucket == 0 ? 8 : 16;
}

struct TuneEntry {
  int lanes;
  float ms[4];  // candidates 4, 8, 16, 32 (0: not tried)
  int64_t sample;
};
static std::mutex g_tune_mu;
static std::map<std::vector<int>, TuneEntry> g_tune;

static std::vector<int> tune_key(const wfa_aligner_t* h, const AlignParams& P, int32_t max_len_sum) {
  return {h->device, metric_class(P.metric), P.format, P.compute_alignment, length_bucket(max_len_sum)};
}

// Lanes per pair for a batch of `todo` pairs (0..todo-1 on the device; the
// samples follow `list`, the batch's cost order, when given).
static int choose_lanes(wfa_aligner_t* h, const AlignParams& P0, int32_t max_len_sum, int64_t todo,
                        cudaStream_t st, bool may_tune, const int64_t* list = nullptr, int32_t max_seq = 0) {
  const int bucket = length_bucket(max_len_sum);
  if (needs_general(P0) || bucket == 3) return 32;
  if (h->lanes_forced) return h->lanes_forced;
  const std::vector<int> key = tune_key(h, P0, max_len_sum);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second.lanes;
  }
  if (!may_tune || todo < kTuneMinPairs) return default_lanes(P0, bucket);
  const int nc = metric_components(P0.metric);
  const int64_t sample = std::min(todo, kTuneSample);
  TuneEntry t{default_lanes(P0, bucket), {0.f, 0.f, 0.f, 0.f}, sample};
  float best = 0.f;
  const int cands[4] = {4, 8, 16, 32};
  for (int ci = 0; ci < 4; ++ci) {
    if (bucket > 0 && cands[ci] < 16) continue;
    float m = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      AlignParams P = P0;
      Round r = first_round(P, nc, max_len_sum, cands[ci], true, max_seq);
      if (launch_round(h, P, r, sample, list, st) != WFA_OK) return default_lanes(P0, bucket);
      if (h->launch_lanes != cands[ci]) break;  // did not fit: ran wider groups
      if (cudaStreamSynchronize(st) != cudaSuccess) return default_lanes(P0, bucket);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, h->ev0, h->ev1);
      m = rep == 0 ? ms : std::min(m, ms);
    }
    if (h->launch_lanes != cands[ci]) continue;
    t.ms[ci] = m;
    if (best == 0.f || m < best) { best = m; t.lanes = cands[ci]; }
  }
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = t;
  return t.lanes;
}

// Runs every pair of a device-resident batch, escalating scratch for pairs
// that need more.  Synchronises `st` to read the retry count.
static int run_device_batch(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* d_results,
                            uint8_t* d_cigars, cudaStream_t st, int32_t max_len_sum,
                            const int64_t* first_list = nullptr, int32_t max_seq = 0) {
  AlignParams P;
  fill_params(h, b, P);
  P.results = d_results;
  P.cigars = d_cigars;
  if (P.compute_alignment && (!d_cigars || !b->cigar_off))
    return fail(h, WFA_ERR_ARGUMENT, "CIGAR output buffers are required in alignment scope");
  const int nc = metric_components(P.metric);
  const int lanes = choose_lanes(h, P, max_len_sum, b->num_pairs, st, true, first_list, max_seq);
  Round r = first_round(P, nc, max_len_sum, lanes, true, max_seq);
  int64_t todo = b->num_pairs;
  const int64_t* list = first_list;
  h->last_kernel_ms = 0.0;
  for (int round = 0; todo > 0; ++round) {
    if (round > 8) return fail(h, WFA_ERR_OOM, "alignment needs more scratch than available");
    int e = launch_round(h, P, r, todo, list, st);
    if (e != WFA_OK) return e;
    if (round == 0) h->last_lanes = h->launch_lanes;
    int32_t retries = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&retries, P.retry_count, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "kernel");
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
    h->last_kernel_ms += ms;
    if (retries == 0) break;
    // Gather the pairs to re-run into a list (double-buffered in pairlist).
    CUDA_TRY(h, h->pairlist.ensure(2 * (size_t)std::max<int64_t>(b->num_pairs, 1) * 8), "pair list");
    int64_t* half0 = h->pairlist.as<int64_t>();
    int64_t* half1 = half0 + b->num_pairs;
    int64_t* out = (list == half0) ? half1 : half0;
    CUDA_TRY(h, cudaMemsetAsync(P.retry_count, 0, 4, st), "memset");
    int tb = 256;
    collect_retries<<<(unsigned)((todo + tb - 1) / tb), tb, 0, st>>>(d_results, list, todo, out,
                                                                     P.retry_count);
    h->launches++;
    CUDA_TRY(h, cudaGetLastError(), "collect retries");
    int32_t got = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&got, P.retry_count, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "collect retries");
    list = out;
    todo = got;
    h->last_reruns += got;
    next_round(r, P, max_len_sum);
  }
  return WFA_OK;
}

// Lanes per pair of a BiWFA launch whose longest pair has n + m = len: a
// team of 8 warps from a few kbp (measured fastest on 2.5-3 kbp pairs and
// on the 1-20 kbp batch), 4 warps for kilobase pairs.
static int biwfa_default_lanes(int32_t len) { return len > 3000 ? 256 : len > 1000 ? 128 : 32; }

// BiWFA batch: the same round structure as run_device_batch with the BiWFA
// kernel and its workspace layout.
static int run_biwfa_batch(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* d_results,
                           uint8_t* d_cigars, cudaStream_t st, int32_t max_len_sum) {
  AlignParams P;
  fill_params(h, b, P);
  P.results = d_results;
  P.cigars = d_cigars;
  if (P.compute_alignment && (!d_cigars || !b->cigar_off))
    return fail(h, WFA_ERR_ARGUMENT, "CIGAR output buffers are required in alignment scope");
  const int cls = metric_class(P.metric);
  const int nc = metric_components(P.metric);
  P.max_len_sum = max_len_sum;
  // Forward/reverse rings are as wide as any wavefront of the launch can be
  // (n + m + 3 cells for the longest pair): a pair re-run for a narrow ring
  // costs its whole alignment again, and ring cells beyond a wavefront's
  // width are never touched.  The base-case ring needs about 2 * 530 + 1
  // cells (a base case ends by score 500 plus one scope).
  ScratchCfg cfg;
  const int32_t wfull = std::max(8, max_len_sum + 3);
  cfg.wmax = wfull;
  int32_t wbase = std::min(cfg.wmax, 1152);
  // Base-case history: every component of scores up to about 550, each at
  // most 2s + 1 cells wide.
  cfg.hist_scores = 1024 * nc;
  cfg.hist_words = (int64_t)nc * 600 * 600;
  const size_t budget = scratch_budget(h);
  const int lanes = bi_lanes_built(h->bi_lanes_forced ? h->bi_lanes_forced : biwfa_default_lanes(max_len_sum),
                                   P.hkind != WFA_HEURISTIC_NONE);
  const int gpb = bi_groups_per_block(lanes);
  const size_t smem = bi_smem_bytes(lanes, P.scope, nc);
  if (smem > 200 * 1024) return fail(h, WFA_ERR_UNSUPPORTED, "wavefront ring too large");
  h->last_lanes = lanes;
  h->launch_lanes = lanes;
  int64_t todo = b->num_pairs;
  const int64_t* list = nullptr;
  h->last_kernel_ms = 0.0;
  // Longest pairs first: the kernel's work queue hands pairs out in list
  // order, so the pairs that take longest start first and the launch does
  // not end waiting on one long pair started late.  The list takes the
  // first third of the pair-list buffer, the re-run lists the other two.
  const int64_t np = b->num_pairs;
  CUDA_TRY(h, h->pairlist.ensure(3 * (size_t)std::max<int64_t>(np, 1) * 8), "pair list");
  int64_t* order_d = h->pairlist.as<int64_t>();
  if (np > 1) {
    std::vector<int32_t> hl((size_t)np), ht((size_t)np);
    CUDA_TRY(h, cudaMemcpyAsync(hl.data(), b->p_len, (size_t)np * 4, cudaMemcpyDeviceToHost, st), "D2H");
    CUDA_TRY(h, cudaMemcpyAsync(ht.data(), b->t_len, (size_t)np * 4, cudaMemcpyDeviceToHost, st), "D2H");
    CUDA_TRY(h, cudaStreamSynchronize(st), "lengths");
    std::vector<int64_t> order((size_t)np);
    for (int64_t i = 0; i < np; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
      return (int64_t)hl[(size_t)x] + ht[(size_t)x] > (int64_t)hl[(size_t)y] + ht[(size_t)y];
    });
    CUDA_TRY(h, cudaMemcpyAsync(order_d, order.data(), (size_t)np * 8, cudaMemcpyHostToDevice, st), "H2D");
    CUDA_TRY(h, cudaStreamSynchronize(st), "pair order");
    list = order_d;
  }
  CUDA_TRY(h, h->counters.ensure(64), "counters");
  P.work_counter = h->counters.as<unsigned long long>();
  P.retry_count = reinterpret_cast<int32_t*>(P.work_counter + 1);
  for (int round = 0; todo > 0; ++round) {
    if (round > 8) return fail(h, WFA_ERR_OOM, "alignment needs more scratch than available");
    const BiLayout L = bi_layout(P.scope, nc, cfg.wmax, wbase, cfg.hist_scores, cfg.hist_words,
                                 max_len_sum, bi_idc_rows(nc, P.e1, P.e2));
    // One wave of resident blocks, no more groups than pairs, and the
    // groups' slices within the scratch budget.
    const int bpsm = std::max(1, occupancy_biwfa(P, cls, lanes, smem));
    int64_t max_groups = (int64_t)h->num_sms * bpsm * gpb;
    int64_t groups = std::max<int64_t>(std::min<int64_t>(max_groups, todo), 1);
    while (groups > 1 && (size_t)groups * L.words * 4 > budget) groups = groups * 3 / 4;
    int blocks = (int)((groups + gpb - 1) / gpb);
    CUDA_TRY(h, h->scratch.ensure((size_t)blocks * gpb * L.words * 4), "scratch");
    P.scratch = h->scratch.as<int32_t>();
    P.warp_words = L.words;
    P.wmax = cfg.wmax;
    P.wmax_base = wbase;
    P.hist_scores = cfg.hist_scores;
    P.hist_words = cfg.hist_words;
    P.pair_list = list;
    P.num_pairs = todo;
    CUDA_TRY(h, cudaMemsetAsync(P.work_counter, 0, 16, st), "memset");
    CUDA_TRY(h, cudaEventRecord(h->ev0, st), "event");
    CUDA_TRY(h, cudaGetLastError(), "an earlier CUDA call of this thread");
    CUDA_TRY(h, launch_biwfa(P, cls, lanes, blocks, smem, st), "BiWFA kernel launch");
    CUDA_TRY(h, cudaEventRecord(h->ev1, st), "event");
    h->launches++;
    int32_t retries = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&retries, P.retry_count, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "kernel");
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
    h->last_kernel_ms += ms;
    if (retries == 0) break;
    int64_t* half0 = order_d + np;
    int64_t* half1 = half0 + np;
    int64_t* out = (list == half0) ? half1 : half0;
    CUDA_TRY(h, cudaMemsetAsync(P.retry_count, 0, 4, st), "memset");
    collect_retries<<<(unsigned)((todo + 255) / 256), 256, 0, st>>>(d_results, list, todo, out, P.retry_count);
    h->launches++;
    CUDA_TRY(h, cudaGetLastError(), "collect retries");
    int32_t got = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&got, P.retry_count, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "collect retries");
    list = out;
    todo = got;
    h->last_reruns += got;
    cfg.wmax = std::min(wfull, cfg.wmax * 2);
    wbase = std::min(cfg.wmax, wbase * 2);
    cfg.hist_scores *= 4;
    cfg.hist_words *= 4;
  }
  return WFA_OK;
}

static int run_batch_kind(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* d_results,
                          uint8_t* d_cigars, cudaStream_t st, int32_t max_len_sum,
                          const int64_t* first_list = nullptr, int32_t max_seq = 0) {
  if (b->span == WFA_SPAN_BIWFA) return run_biwfa_batch(h, b, d_results, d_cigars, st, max_len_sum);
  return run_device_batch(h, b, d_results, d_cigars, st, max_len_sum, first_list, max_seq);
}

// Cost ordering (wfa_order.cu) for lean batches of short pairs: the lane
// groups of a warp then get pairs of similar cost.  Batches below
// kSortMinPairs run in input order.
static constexpr int64_t kSortMinPairs = 16384;

static bool orders_batch(const wfa_aligner_t* h, const wfa_batch_t* b) {
  if (b->span == WFA_SPAN_BIWFA || b->num_pairs < kSortMinPairs) return false;
  AlignParams P;
  fill_params(h, b, P);
  return !needs_general(P);
}

// Layout of h->order for n pairs and `parts` separately ordered ranges:
// keys (u16), pair lists (i64), then per range kOrderStride ints: a
// histogram and a fill counter array (kOrderBins each) and a longest-pair
// word.
static constexpr int64_t kOrderStride = 2 * kOrderBins + 32;
struct OrderBufs {
  uint16_t* keys;
  int64_t* list;
  int32_t* hist;  // [parts][kOrderStride]
};
static int order_bufs(wfa_aligner_t* h, int64_t n, int64_t parts, OrderBufs* o) {
  const size_t keys = ((size_t)n * 2 + 15) & ~(size_t)15;
  const size_t list = (size_t)n * 8;
  const size_t hist = (size_t)parts * kOrderStride * 4;
  CUDA_TRY(h, h->order.ensure(keys + list + hist), "ordering buffers");
  char* base = h->order.as<char>();
  o->keys = reinterpret_cast<uint16_t*>(base);
  o->list = reinterpret_cast<int64_t*>(base + keys);
  o->hist = reinterpret_cast<int32_t*>(base + keys + list);
  return WFA_OK;
}

// ---------------------------------------------------------------------------
// Batch without allocation: the scratch is the fixed array of wfa_noalloc.cu.
// Its layout (int32 words): a 64-word header (work counter, retry count,
// longest n + m, retry-list fill), the retry list (int64 pair indices), then
// the per-warp slices.
// ---------------------------------------------------------------------------
static constexpr int64_t kNaHeaderWords = 64;
static constexpr int32_t kNaListCap = 65536;  // pairs re-run per round
static constexpr int64_t kNaSliceOff = kNaHeaderWords + 2 * (int64_t)kNaListCap;
static constexpr int64_t kNaSliceWords = (int64_t)(kNoAllocScratchBytes / 4) - kNaSliceOff;

// Every pair of 0..n-1 still marked for re-running, up to `cap` of them, into
// out[]; *count ends as the number of such pairs (it may exceed cap).
__global__ void collect_retries_capped(const wfa_result_t* res, int64_t n, int64_t* out,
                                       int32_t* count, int32_t cap) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || res[i].status != kStatusRetry) return;
  int32_t slot = atomicAdd(count, 1);
  if (slot < cap) out[slot] = i;
}

// The rounds of run_device_batch over the fixed array: the first round gives
// each warp a small M history so that many warps fit; pairs that need more
// are gathered (at most kNaListCap per round) and re-run with larger slices,
// until a slice no longer fits a block's warps in the array.
static int run_noalloc_batch(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* d_results,
                             uint8_t* d_cigars, cudaStream_t st, int32_t* base, int32_t max_len_sum) {
  AlignParams P;
  fill_params(h, b, P);
  P.results = d_results;
  P.cigars = d_cigars;
  if (P.compute_alignment && (!d_cigars || !b->cigar_off))
    return fail(h, WFA_ERR_ARGUMENT, "CIGAR output buffers are required in alignment scope");
  const int cls = metric_class(P.metric);
  const int nc = metric_components(P.metric);
  unsigned long long* work = reinterpret_cast<unsigned long long*>(base);
  int32_t* retry = base + 2;
  int32_t* fill = base + 4;
  int64_t* list = reinterpret_cast<int64_t*>(base + kNaHeaderWords);
  // Whole warps per pair, and no spill ring: a row wider than the shared
  // memory slot re-runs the pair with the ring in its slice.
  Round r = first_round(P, nc, max_len_sum, 32, false);
  if (P.compute_alignment && !P.piggyback) {
    r.cfg.hist_scores = 256;
    r.cfg.hist_words = 4096;
  }
  int64_t todo = b->num_pairs, pending = 0;
  int grown = 0;
  const int64_t* lst = nullptr;
  h->last_kernel_ms = 0.0;
  for (;;) {
    int64_t warp_words = 0;
    const SmemLayout L = round_layout(P, r, nc, &warp_words);
    if (L.total > 200 * 1024) return fail(h, WFA_ERR_UNSUPPORTED, "wavefront ring too large");
    const int occ = round_occupancy(h, P, cls, r.lanes, L.total);
    const int64_t fit_blocks = kNaSliceWords / (warp_words * kWarpsPerBlock);
    if (fit_blocks < 1)
      return fail(h, WFA_ERR_OOM, "an alignment needs more scratch than the fixed no-allocation "
                                  "array holds (use wfa_batch_align_device)");
    int64_t warps = std::min<int64_t>((int64_t)h->num_sms * occ * kWarpsPerBlock, todo);
    int64_t blocks = std::min<int64_t>((std::max<int64_t>(warps, 1) + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                       fit_blocks);
    P.scratch = base + kNaSliceOff;
    P.warp_words = warp_words;
    P.work_counter = work;
    P.retry_count = retry;
    P.pair_list = lst;
    P.num_pairs = todo;
    CUDA_TRY(h, cudaMemsetAsync(base, 0, 16, st), "memset");
    CUDA_TRY(h, cudaEventRecord(h->ev0, st), "event");
    CUDA_TRY(h, cudaGetLastError(), "an earlier CUDA call of this thread");
    CUDA_TRY(h, launch_unialign(P, cls, r.lanes, (int)blocks, L.total, st), "kernel launch");
    CUDA_TRY(h, cudaEventRecord(h->ev1, st), "event");
    h->launches++;
    int32_t retries = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&retries, retry, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "kernel");
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
    h->last_kernel_ms += ms;
    if (retries == 0 && pending == 0) break;
    // Pairs that failed in this round need larger slices; pairs left over
    // from an earlier gathering are re-run at the current size first.
    if (retries > 0) {
      if (++grown > 16) return fail(h, WFA_ERR_OOM, "alignment needs more scratch than available");
      next_round(r, P, max_len_sum);
    }
    CUDA_TRY(h, cudaMemsetAsync(fill, 0, 4, st), "memset");
    const int64_t n = b->num_pairs;
    collect_retries_capped<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_results, n, list, fill,
                                                                        kNaListCap);
    h->launches++;
    CUDA_TRY(h, cudaGetLastError(), "collect retries");
    int32_t got = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&got, fill, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "collect retries");
    if (got == 0) break;
    todo = std::min(got, kNaListCap);
    if (retries > 0) h->last_reruns += retries;
    pending = got - todo;
    lst = list;
  }
  return WFA_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int wfa_penalties_check(wfa_metric_t metric, const wfa_penalties_t* penalties) {
  AlignParams P{};
  return set_penalties((int)metric, penalties, P);
}

wfa_aligner_t* wfa_aligner_create(wfa_metric_t metric, const wfa_penalties_t* penalties,
                                  int device, int* err) {
  AlignParams P{};
  int r = set_penalties((int)metric, penalties, P);
  if (r != WFA_OK) {
    if (err) *err = r;
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || device < 0 || device >= ndev) {
    if (err) *err = WFA_ERR_NO_DEVICE;
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    if (err) *err = WFA_ERR_CUDA;
    return nullptr;
  }
  wfa_aligner_t* h = new wfa_aligner();
  h->device = device;
  h->pen = P;
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->s_cig, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    delete h;
    if (err) *err = WFA_ERR_CUDA;
    return nullptr;
  }
  for (DevBuf* b : {&h->seq, &h->poff, &h->plen, &h->toff, &h->tlen, &h->coff, &h->results,
                    &h->cigars, &h->dense, &h->scratch, &h->counters, &h->pairlist, &h->chunkinfo,
                    &h->order, &h->checks})
    b->st = h->stream;
#ifdef WFA_DEVICE_CHECKS
  if (h->checks.ensure(16) != cudaSuccess || cudaMemset(h->checks.p, 0, 16) != cudaSuccess) {
    wfa_aligner_destroy(h);
    if (err) *err = WFA_ERR_CUDA;
    return nullptr;
  }
#endif
  // Events made now rather than by the first batches: creating an event
  // waits for the work running on the device, which beside a resident
  // stream's kernel (running until it has been idle for about a second)
  // would hold a batch that long.
  if (event_pool(h, 32) != cudaSuccess || timing_events(h, 16) != cudaSuccess) {
    wfa_aligner_destroy(h);
    if (err) *err = WFA_ERR_CUDA;
    return nullptr;
  }
  if (err) *err = WFA_OK;
  return h;
}

void wfa_aligner_destroy(wfa_aligner_t* h) {
  if (!h) return;
  if (h->async_worker.joinable()) {  // finish the submitted batches first
    {
      std::lock_guard<std::mutex> lock(h->async_mu);
      h->async_stop = true;
    }
    h->async_cv.notify_all();
    h->async_worker.join();
  }
  cudaSetDevice(h->device);
  for (cudaStream_t x : {h->stream, h->s_in, h->s_out, h->s_cig})
    if (x) cudaStreamSynchronize(x);
  for (DevBuf* b : {&h->seq, &h->poff, &h->plen, &h->toff, &h->tlen, &h->coff, &h->results,
                    &h->cigars, &h->dense, &h->scratch, &h->counters, &h->pairlist, &h->chunkinfo,
                    &h->order, &h->checks})
    b->release();
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->hinfo) cudaFreeHost(h->hinfo);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
  for (cudaEvent_t e : h->evtime) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->s_in) cudaStreamDestroy(h->s_in);
  if (h->s_out) cudaStreamDestroy(h->s_out);
  if (h->s_cig) cudaStreamDestroy(h->s_cig);
  delete h;
}

int wfa_set_memory_mode(wfa_aligner_t* h, wfa_memory_t mode) {
  if (!h || mode < WFA_MEMORY_HIGH || mode > WFA_MEMORY_LOW) return WFA_ERR_ARGUMENT;
  h->memory_mode = mode;
  return WFA_OK;
}
int wfa_set_max_memory_compact(wfa_aligner_t* h, uint64_t bytes) {
  if (!h) return WFA_ERR_ARGUMENT;
  h->max_memory_compact = bytes;
  return WFA_OK;
}
int wfa_set_max_alignment_steps(wfa_aligner_t* h, int32_t s) {
  if (!h) return WFA_ERR_ARGUMENT;
  h->max_steps = s;
  return WFA_OK;
}
int wfa_set_alignment_scope(wfa_aligner_t* h, wfa_scope_t scope) {
  if (!h || (scope != WFA_SCOPE_SCORE && scope != WFA_SCOPE_ALIGNMENT)) return WFA_ERR_ARGUMENT;
  h->scope = scope;
  return WFA_OK;
}
int wfa_set_alignment_free_ends(wfa_aligner_t* h, int32_t p0, int32_t pf, int32_t t0, int32_t tf) {
  if (!h) return WFA_ERR_ARGUMENT;  // src/aligner.rs:563-576
  h->span = WFA_SPAN_ENDSFREE;
  h->extension = 0;
  h->p0 = p0; h->pf = pf; h->t0 = t0; h->tf = tf;
  return WFA_OK;
}
int wfa_set_alignment_extension(wfa_aligner_t* h) {
  if (!h) return WFA_ERR_ARGUMENT;  // src/aligner.rs:582-585
  h->span = WFA_SPAN_ENDSFREE;
  h->extension = 1;
  return WFA_OK;
}
int wfa_set_alignment_end_to_end(wfa_aligner_t* h) {
  if (!h) return WFA_ERR_ARGUMENT;  // src/aligner.rs:595-603
  h->span = WFA_SPAN_END2END;
  h->extension = 0;
  h->p0 = h->pf = h->t0 = h->tf = 0;
  return WFA_OK;
}
int wfa_set_compat(wfa_aligner_t* h, wfa_compat_t c) {
  if (!h || (c != WFA_COMPAT_C && c != WFA_COMPAT_CORRECTED)) return WFA_ERR_ARGUMENT;
  h->compat = c;
  return WFA_OK;
}
int wfa_set_heuristic(wfa_aligner_t* h, wfa_heuristic_kind_t kind, int32_t p0, int32_t p1,
                      int32_t p2) {
  if (!h || kind < WFA_HEURISTIC_NONE || kind > WFA_HEURISTIC_BANDED_ADAPTIVE) return WFA_ERR_ARGUMENT;
  h->hkind = kind;
  h->hp0 = p0; h->hp1 = p1; h->hp2 = p2;
  return WFA_OK;
}

// One pair through the batch kernel (plain per-call form): one host->device
// copy (sequences and metadata in one pinned staging buffer), one launch, the
// result record and CIGAR slot copied back, one synchronisation.  A pair that
// needs more scratch than the first configuration is re-run by the batch
// driver.
static int32_t align_plain(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t,
                           int32_t m, int span, bool packed) {
  if (!h || n < 0 || m < 0 || (n > 0 && !p) || (m > 0 && !t)) return WFA_ERR_ARGUMENT;
  h->last_err = WFA_OK;
  h->status = WFA_STATUS_OOM;
  h->cigar.clear();
  int saved_span = h->span;
  h->span = span;
  int r = check_supported(h, span == WFA_SPAN_BIWFA);
  h->span = saved_span;
  if (r != WFA_OK) return r;
  cudaSetDevice(h->device);
  cudaStream_t st = h->stream;
  // Staging layout: [meta 64 B][pattern, 16-aligned][text, 16-aligned][pad].
  struct Meta { int64_t poff, toff, coff; int32_t plen, tlen; };
  const size_t pbytes = packed ? ((size_t)n + 3) / 4 : (size_t)n;
  const size_t tbytes = packed ? ((size_t)m + 3) / 4 : (size_t)m;
  const size_t seq0 = 64;
  const size_t toff_b = (pbytes + 15) & ~(size_t)15;
  const size_t total = seq0 + toff_b + ((tbytes + 15) & ~(size_t)15) + 16;
  const int64_t cap = 2 * ((int64_t)n + m) + 1;
  if (total > h->pinned_cap) {
    if (h->pinned) cudaFreeHost(h->pinned);
    h->pinned = nullptr;
    h->pinned_cap = 0;
    size_t want = std::max(total, (size_t)1 << 16);
    CUDA_TRY(h, cudaMallocHost(&h->pinned, want), "pinned staging");
    h->pinned_cap = want;
  }
  std::memset(h->pinned, 0, total);
  Meta meta;
  meta.poff = 0;
  meta.toff = packed ? (int64_t)(toff_b / 4) : (int64_t)toff_b;
  meta.coff = 0;
  meta.plen = n;
  meta.tlen = m;
  std::memcpy(h->pinned, &meta, sizeof meta);
  if (pbytes) std::memcpy(h->pinned + seq0, p, pbytes);
  if (tbytes) std::memcpy(h->pinned + seq0 + toff_b, t, tbytes);
  CUDA_TRY(h, h->seq.ensure(total), "seq");
  CUDA_TRY(h, h->results.ensure(sizeof(wfa_result_t)), "results");
  CUDA_TRY(h, h->cigars.ensure((size_t)cap), "cigars");
  CUDA_TRY(h, cudaMemcpyAsync(h->seq.p, h->pinned, total, cudaMemcpyHostToDevice, st), "H2D");
  const char* mb = h->seq.as<char>();
  wfa_batch_t b;
  b.format = packed ? WFA_SEQ_PACKED2 : WFA_SEQ_ASCII;
  b.span = span;
  b.num_pairs = 1;
  b.seq = mb + seq0;
  b.seq_bytes = (int64_t)(total - seq0);
  b.p_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, poff));
  b.t_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, toff));
  b.cigar_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, coff));
  b.p_len = reinterpret_cast<const int32_t*>(mb + offsetof(Meta, plen));
  b.t_len = reinterpret_cast<const int32_t*>(mb + offsetof(Meta, tlen));
  b.cigar_bytes = cap;
  AlignParams P;
  fill_params(h, &b, P);
  P.results = h->results.as<wfa_result_t>();
  P.cigars = h->cigars.as<uint8_t>();
  const bool aln = P.compute_alignment != 0;
  if (span == WFA_SPAN_BIWFA) {
    r = run_biwfa_batch(h, &b, P.results, P.cigars, st, n + m);
  } else {
    Round rd = first_round(P, metric_components(P.metric), n + m);
    r = launch_round(h, P, rd, 1, nullptr, st);
  }
  if (r != WFA_OK) return r;
  wfa_result_t res;
  uint8_t* hbuf = h->pinned;  // reuse staging for the way back
  const size_t back = sizeof(wfa_result_t) + (aln ? (size_t)cap : 0);
  if (back > h->pinned_cap) {
    CUDA_TRY(h, cudaStreamSynchronize(st), "sync");
    cudaFreeHost(h->pinned);
    h->pinned = nullptr;
    h->pinned_cap = 0;
    CUDA_TRY(h, cudaMallocHost(&h->pinned, back), "pinned staging");
    h->pinned_cap = back;
    hbuf = h->pinned;
  }
  CUDA_TRY(h, cudaMemcpyAsync(hbuf, h->results.p, sizeof res, cudaMemcpyDeviceToHost, st), "D2H");
  if (aln)
    CUDA_TRY(h, cudaMemcpyAsync(hbuf + sizeof res, h->cigars.p, (size_t)cap, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  std::memcpy(&res, hbuf, sizeof res);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_kernel_ms = ms;
  if (res.status == kStatusRetry) {
    r = run_device_batch(h, &b, h->results.as<wfa_result_t>(), h->cigars.as<uint8_t>(), st, n + m);
    if (r != WFA_OK) return r;
    CUDA_TRY(h, cudaMemcpyAsync(hbuf, h->results.p, sizeof res, cudaMemcpyDeviceToHost, st), "D2H");
    if (aln)
      CUDA_TRY(h, cudaMemcpyAsync(hbuf + sizeof res, h->cigars.p, (size_t)cap, cudaMemcpyDeviceToHost, st), "D2H");
    CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
    std::memcpy(&res, hbuf, sizeof res);
  }
  if (res.cigar_length > 0) {
    const uint8_t* ops = hbuf + sizeof res + res.cigar_begin;
    h->cigar.assign(ops, ops + res.cigar_length);
  }
  h->status = res.status;
  h->cigar_score = res.cigar_score;
  h->end_v = res.end_v;
  h->end_h = res.end_h;
  h->end_score = res.end_score;
  h->end_k = res.end_k;
  h->end_offset = res.end_offset;
  return res.score;
}

int32_t wfa_align_end2end(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  return align_plain(h, p, n, t, m, WFA_SPAN_END2END, false);
}
int32_t wfa_align_endsfree(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  if (h && h->extension) {  // src/aligner.rs:713-718
    h->p0 = 0; h->pf = n; h->t0 = 0; h->tf = m;
  }
  return align_plain(h, p, n, t, m, h ? h->span : 0, false);
}
int32_t wfa_align_packed2bits(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  return align_plain(h, p, n, t, m, WFA_SPAN_END2END, true);
}
int32_t wfa_align_biwfa(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  if (!h) return WFA_ERR_ARGUMENT;
  h->scope = WFA_SCOPE_ALIGNMENT;  // align_biwfa sets ComputeAlignment (src/aligner.rs:2565)
  return align_plain(h, p, n, t, m, WFA_SPAN_BIWFA, false);
}
int32_t wfa_align_biwfa_score(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  if (!h) return WFA_ERR_ARGUMENT;
  int saved = h->scope;
  h->scope = WFA_SCOPE_SCORE;
  int32_t r = align_plain(h, p, n, t, m, WFA_SPAN_BIWFA, false);
  h->scope = saved;
  return r;
}
int32_t wfa_align_lambda(wfa_aligner_t* h, int (*)(int32_t, int32_t, void*), void*, int32_t, int32_t) {
  return fail(h, WFA_ERR_UNSUPPORTED, "lambda sequences need a host callback per comparison");
}

wfa_status_t wfa_status(const wfa_aligner_t* h) { return h ? (wfa_status_t)h->status : WFA_STATUS_OOM; }
int wfa_cigar(const wfa_aligner_t* h, const uint8_t** ops, int32_t* len, int32_t* score,
              int32_t* ev, int32_t* eh) {
  if (!h) return WFA_ERR_ARGUMENT;
  if (ops) *ops = h->cigar.empty() ? nullptr : h->cigar.data();
  if (len) *len = (int32_t)h->cigar.size();
  if (score) *score = h->cigar_score;
  if (ev) *ev = h->end_v;
  if (eh) *eh = h->end_h;
  return WFA_OK;
}
int wfa_alignment_end_pos(const wfa_aligner_t* h, int32_t* s, int32_t* k, int32_t* o) {
  if (!h) return WFA_ERR_ARGUMENT;
  if (s) *s = h->end_score;
  if (k) *k = h->end_k;
  if (o) *o = h->end_offset;
  return WFA_OK;
}
int wfa_last_error(const wfa_aligner_t* h) { return h ? h->last_err : WFA_ERR_ARGUMENT; }
const char* wfa_last_error_string(const wfa_aligner_t* h) { return h ? h->err_str.c_str() : "null handle"; }
int64_t wfa_kernel_launches(const wfa_aligner_t* h) { return h ? h->launches : 0; }
int64_t wfa_device_check_failures(wfa_aligner_t* h) {
#ifdef WFA_DEVICE_CHECKS
  if (!h) return WFA_ERR_ARGUMENT;
  int32_t v = 0;
  cudaSetDevice(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
      cudaMemcpy(&v, h->checks.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return WFA_ERR_CUDA;
  return v;
#else
  return h ? -1 : WFA_ERR_ARGUMENT;
#endif
}
int64_t wfa_last_rerun_pairs(const wfa_aligner_t* h) { return h ? h->last_reruns : 0; }
int wfa_set_lanes_per_pair(wfa_aligner_t* h, int32_t lanes) {
  if (!h || !(lanes == 0 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32)) return WFA_ERR_ARGUMENT;
  h->lanes_forced = lanes;
  return WFA_OK;
}
int wfa_set_biwfa_lanes(wfa_aligner_t* h, int32_t lanes) {
  if (!h || !(lanes == 0 || lanes == 32 || lanes == 128 || lanes == 256 || lanes == 512)) return WFA_ERR_ARGUMENT;
  h->bi_lanes_forced = lanes;
  return WFA_OK;
}
int32_t wfa_last_lanes_per_pair(const wfa_aligner_t* h) { return h ? h->last_lanes : 0; }
int64_t wfa_last_slice_bytes(const wfa_aligner_t* h) { return h ? h->last_slice_bytes : 0; }
int32_t wfa_autotune_report(char* out, int32_t cap) {
  std::string r;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    char line[256];
    for (const auto& kv : g_tune) {
      const std::vector<int>& k = kv.first;
      const TuneEntry& t = kv.second;
      std::snprintf(line, sizeof line,
                    "device %d class %d format %d cigar %d bucket %d: lanes %d (sample %lld pairs; "
                    "ms 4:%.3f 8:%.3f 16:%.3f 32:%.3f)\n",
                    k[0], k[1], k[2], k[3], k[4], t.lanes, (long long)t.sample, t.ms[0], t.ms[1], t.ms[2],
                    t.ms[3]);
      r += line;
    }
  }
  if (out && cap > 0) {
    int32_t c = std::min<int32_t>((int32_t)r.size(), cap - 1);
    std::memcpy(out, r.data(), (size_t)c);
    out[c] = 0;
  }
  return (int32_t)r.size();
}
double wfa_last_kernel_ms(const wfa_aligner_t* h) { return h ? h->last_kernel_ms : 0.0; }

static int batch_common(wfa_aligner_t* h, const wfa_batch_t* b) {
  if (!h || !b || b->num_pairs < 0 || !b->seq || !b->p_off || !b->p_len || !b->t_off || !b->t_len)
    return WFA_ERR_ARGUMENT;
  if (b->format != WFA_SEQ_ASCII && b->format != WFA_SEQ_PACKED2) return WFA_ERR_ARGUMENT;
  if (b->span != WFA_SPAN_END2END && b->span != WFA_SPAN_ENDSFREE && b->span != WFA_SPAN_BIWFA)
    return WFA_ERR_ARGUMENT;
  h->last_err = WFA_OK;
  h->last_reruns = 0;
  int saved = h->span;
  h->span = b->span;
  int r = check_supported(h, b->span == WFA_SPAN_BIWFA);
  h->span = saved;
  return r;
}

int wfa_batch_align_device(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results,
                           uint8_t* cigars, void* stream) {
  int r = batch_common(h, b);
  if (r != WFA_OK) return r;
  if (b->num_pairs == 0) return WFA_OK;
  cudaSetDevice(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  CUDA_TRY(h, h->counters.ensure(64), "counters");
  int32_t* d_max = reinterpret_cast<int32_t*>(h->counters.as<char>() + 32);
  CUDA_TRY(h, cudaMemsetAsync(d_max, 0, 8, st), "memset");
  const bool order = orders_batch(h, b);
  OrderBufs ob{};
  if (order) {
    // The longest pair, the cost keys and the ordered list in one pass (one
    // cooperative launch), before the host waits; the list goes unused if the
    // batch turns out to hold long pairs.
    if (int e = order_bufs(h, b->num_pairs, 1, &ob)) return e;
    CUDA_TRY(h, cudaMemsetAsync(ob.hist, 0, kOrderStride * 4, st), "memset");
    int nl = 0;
    CUDA_TRY(h, launch_order(static_cast<const uint8_t*>(b->seq), b->format == WFA_SEQ_PACKED2, b->p_off, b->p_len,
                             b->t_off, b->t_len, b->num_pairs, h->num_sms, d_max, ob.keys, ob.hist,
                             ob.hist + kOrderBins, ob.list, st, &nl),
             "cost order");
    h->launches += nl;
  } else {
    max_lengths<<<256, 256, 0, st>>>(b->p_len, b->t_len, b->num_pairs, d_max);
    CUDA_TRY(h, cudaGetLastError(), "max lengths");
    h->launches++;
  }
  int32_t mxs[2] = {0, 0};
  CUDA_TRY(h, cudaMemcpyAsync(mxs, d_max, 8, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "max lengths");
  const int32_t mx = mxs[0];
  const int64_t* first = order && length_bucket(mx) <= 2 ? ob.list : nullptr;
  return run_batch_kind(h, b, results, cigars, st, mx, first, mxs[1]);
}

// The device-buffer batch on the fixed array of wfa_noalloc.cu: no cudaMalloc,
// cudaFree or other allocation on any path.  Declared with its limits in
// wfa_b200.h.
int wfa_batch_align_device_noalloc(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results,
                                   uint8_t* cigars, void* stream) {
  int r = batch_common(h, b);
  if (r != WFA_OK) return r;
  if (b->span == WFA_SPAN_BIWFA)
    return fail(h, WFA_ERR_UNSUPPORTED, "the no-allocation batch runs end-to-end and ends-free spans only");
  if (b->num_pairs == 0) return WFA_OK;
  CUDA_TRY(h, cudaSetDevice(h->device), "set device");
  int32_t* base = nullptr;
  CUDA_TRY(h, noalloc_scratch(h->device, &base), "address of the no-allocation scratch array");
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  int32_t* d_max = base + 6;  // header words 6, 7: longest n + m, longest sequence
  CUDA_TRY(h, cudaMemsetAsync(base, 0, kNaHeaderWords * 4, st), "memset");
  max_lengths<<<256, 256, 0, st>>>(b->p_len, b->t_len, b->num_pairs, d_max);
  h->launches++;
  CUDA_TRY(h, cudaGetLastError(), "max lengths");
  int32_t mx = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&mx, d_max, 4, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "max lengths");
  if (mx > WFA_NOALLOC_MAX_LEN_SUM)
    return fail(h, WFA_ERR_ARGUMENT, "a pair has p_len + t_len above WFA_NOALLOC_MAX_LEN_SUM (4096), "
                                     "the limit of the no-allocation batch");
  return run_noalloc_batch(h, b, results, cigars, st, base, mx);
}

// Host-buffer batch without pipelining (BiWFA): copy in, align, dense CIGARs out.
static int batch_align_simple(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results,
                              uint8_t* cigars) {
  const int64_t n = b->num_pairs;
  const bool aln = h->scope == WFA_SCOPE_ALIGNMENT;
  cudaStream_t st = h->stream;
  int32_t mx = 0;
  int64_t slot_total = 0;
  std::vector<int64_t> slot_off(aln ? (size_t)n : 0);
  for (int64_t i = 0; i < n; ++i) {
    int32_t s = b->p_len[i] + b->t_len[i];
    mx = std::max(mx, s);
    if (aln) { slot_off[(size_t)i] = slot_total; slot_total += 2 * (int64_t)s + 1; }
  }
  size_t seq_bytes = ((size_t)b->seq_bytes + 15) & ~(size_t)15;
  CUDA_TRY(h, h->seq.ensure(seq_bytes + 16), "seq");
  CUDA_TRY(h, h->poff.ensure((size_t)n * 8), "p_off");
  CUDA_TRY(h, h->toff.ensure((size_t)n * 8), "t_off");
  CUDA_TRY(h, h->plen.ensure((size_t)n * 4), "p_len");
  CUDA_TRY(h, h->tlen.ensure((size_t)n * 4), "t_len");
  CUDA_TRY(h, h->results.ensure((size_t)n * sizeof(wfa_result_t)), "results");
  CUDA_TRY(h, cudaMemcpyAsync(h->seq.p, b->seq, (size_t)b->seq_bytes, cudaMemcpyHostToDevice, st), "H2D");
  CUDA_TRY(h, cudaMemcpyAsync(h->poff.p, b->p_off, (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
  CUDA_TRY(h, cudaMemcpyAsync(h->toff.p, b->t_off, (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
  CUDA_TRY(h, cudaMemcpyAsync(h->plen.p, b->p_len, (size_t)n * 4, cudaMemcpyHostToDevice, st), "H2D");
  CUDA_TRY(h, cudaMemcpyAsync(h->tlen.p, b->t_len, (size_t)n * 4, cudaMemcpyHostToDevice, st), "H2D");
  wfa_batch_t d = *b;
  d.seq = h->seq.p;
  d.seq_bytes = (int64_t)seq_bytes;
  d.p_off = h->poff.as<int64_t>(); d.t_off = h->toff.as<int64_t>();
  d.p_len = h->plen.as<int32_t>(); d.t_len = h->tlen.as<int32_t>();
  d.cigar_off = nullptr;
  if (aln) {
    CUDA_TRY(h, h->coff.ensure((size_t)n * 8), "cigar_off");
    CUDA_TRY(h, h->cigars.ensure((size_t)slot_total + 16), "cigar slots");
    CUDA_TRY(h, cudaMemcpyAsync(h->coff.p, slot_off.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
    d.cigar_off = h->coff.as<int64_t>();
    d.cigar_bytes = slot_total;
  }
  int r = run_batch_kind(h, &d, h->results.as<wfa_result_t>(), aln ? h->cigars.as<uint8_t>() : nullptr, st, mx);
  if (r != WFA_OK) return r;
  CUDA_TRY(h, cudaMemcpyAsync(results, h->results.p, (size_t)n * sizeof(wfa_result_t), cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  if (!aln) return WFA_OK;
  std::vector<int64_t> dst((size_t)n);
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) { dst[(size_t)i] = total; total += results[i].cigar_length; }
  CUDA_TRY(h, h->dense.ensure((size_t)total + 16), "dense cigars");
  CUDA_TRY(h, h->pairlist.ensure((size_t)n * 8), "offsets");
  CUDA_TRY(h, cudaMemcpyAsync(h->pairlist.p, dst.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
  compact_cigars<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(
      h->results.as<wfa_result_t>(), d.cigar_off, h->cigars.as<uint8_t>(), h->pairlist.as<int64_t>(),
      h->dense.as<uint8_t>(), n);
  h->launches++;
  CUDA_TRY(h, cudaGetLastError(), "compact cigars");
  CUDA_TRY(h, cudaMemcpyAsync(cigars, h->dense.p, (size_t)total, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  for (int64_t i = 0; i < n; ++i) results[i].cigar_begin = (int32_t)dst[(size_t)i];
  return WFA_OK;
}

// Host-buffer batch, pipelined in chunks of pairs: while chunk c aligns on
// the compute stream, chunk c+1's inputs are copied in and chunk c-1's packed
// CIGARs (packed on the device right after its alignment: a prefix sum of
// the CIGAR lengths, then the compaction) are copied out with its results.
// The host only waits for each chunk's results to issue the copy of its
// packed CIGAR bytes.  CIGARs are
// packed densely in input order; results[i].cigar_begin is the offset of
// pair i's ops in `cigars`.  Pairs that need more scratch than the first
// configuration are re-run at the end by the batch driver.
int wfa_batch_align(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results, uint8_t* cigars) {
  int r = batch_common(h, b);
  if (r != WFA_OK) return r;
  if (!results) return WFA_ERR_ARGUMENT;
  const int64_t n = b->num_pairs;
  if (n == 0) return WFA_OK;
  const bool aln = h->scope == WFA_SCOPE_ALIGNMENT;
  if (aln && !cigars) return WFA_ERR_ARGUMENT;
  cudaSetDevice(h->device);
  if (b->span == WFA_SPAN_BIWFA) return batch_align_simple(h, b, results, cigars);
  cudaStream_t sc = h->stream, si = h->s_in, so = h->s_out;
  // Chunks of `chunk` pairs, the first and last a quarter of that: a short
  // first chunk starts the device sooner, a short last one leaves less to
  // copy out after the last alignment.  Chunks of half the batch (up to
  // 524,288 pairs) keep each launch long enough for narrow lane groups (on
  // the 1M-pair short-read batch: 4.96 ms of kernel time in chunks of a half,
  // 7.38 ms in chunks of an eighth).
  const int64_t chunk = std::max<int64_t>(65536, std::min<int64_t>(524288, (n + 1) / 2));
  std::vector<int64_t> bnd{0};
  {
    const int64_t edge = std::max<int64_t>(chunk / 4, 1);
    int64_t at = std::min(n, edge);
    bnd.push_back(at);
    while (n - at > edge) {
      at += std::min(chunk, n - at - edge);
      bnd.push_back(at);
    }
    if (at < n) bnd.push_back(n);
  }
  const int64_t nchunks = (int64_t)bnd.size() - 1;
  const bool packed = b->format == WFA_SEQ_PACKED2;

  // Per chunk: sequence byte range, longest pair, CIGAR slot bytes -- one
  // pass over the host arrays, split across host threads.
  std::vector<ChunkInfo> ci_info((size_t)nchunks);
  scan_chunks(b, n, bnd, packed, aln, ci_info);
  std::vector<int64_t> c_slot0((size_t)nchunks + 1, 0);
  for (int64_t ci = 0; ci < nchunks; ++ci)
    c_slot0[(size_t)ci + 1] = c_slot0[(size_t)ci] + ci_info[(size_t)ci].slots;
  const int64_t slot_total = c_slot0[(size_t)nchunks];

  size_t seq_bytes = ((size_t)b->seq_bytes + 15) & ~(size_t)15;
  CUDA_TRY(h, h->seq.ensure(seq_bytes + 16), "seq");
  CUDA_TRY(h, h->poff.ensure((size_t)n * 8), "p_off");
  CUDA_TRY(h, h->toff.ensure((size_t)n * 8), "t_off");
  CUDA_TRY(h, h->plen.ensure((size_t)n * 4), "p_len");
  CUDA_TRY(h, h->tlen.ensure((size_t)n * 4), "t_len");
  CUDA_TRY(h, h->results.ensure((size_t)n * sizeof(wfa_result_t)), "results");
  if (aln) {
    CUDA_TRY(h, h->coff.ensure((size_t)n * 8), "cigar_off");
    CUDA_TRY(h, h->cigars.ensure((size_t)slot_total + 16), "cigar slots");
    CUDA_TRY(h, h->dense.ensure((size_t)slot_total + 16), "dense cigars");
    CUDA_TRY(h, h->pairlist.ensure((size_t)n * 8), "dense offsets");
  }
  // Per chunk on the device: work/retry counters (2 words) and the dense
  // CIGAR range [begin, end) (2 words), plus the running dense total.
  const int64_t ntiles = (chunk + kScanTile - 1) / kScanTile;
  CUDA_TRY(h, h->chunkinfo.ensure((size_t)(4 * nchunks + 1 + ntiles) * 8), "chunk counters");
  CUDA_TRY(h, host_info(h, (size_t)nchunks * 4), "pinned chunk info");
  CUDA_TRY(h, event_pool(h, 4 * (size_t)nchunks), "events");
  CUDA_TRY(h, timing_events(h, 2 * (size_t)nchunks), "events");
  cudaEvent_t* ev_in = h->evpool.data();
  cudaEvent_t* ev_k = ev_in + nchunks;
  cudaEvent_t* ev_x = ev_k + nchunks;
  cudaEvent_t* ev_res = ev_x + nchunks;
  uint8_t* dseq = h->seq.as<uint8_t>();
  int64_t *dpo = h->poff.as<int64_t>(), *dto = h->toff.as<int64_t>();
  int32_t *dpl = h->plen.as<int32_t>(), *dtl = h->tlen.as<int32_t>();
  wfa_result_t* dres = h->results.as<wfa_result_t>();
  int64_t* dco = aln ? h->coff.as<int64_t>() : nullptr;
  int64_t* ddst = aln ? h->pairlist.as<int64_t>() : nullptr;
  unsigned long long* dctr = h->chunkinfo.as<unsigned long long>();  // [chunk][work, retry]
  int64_t* drange = reinterpret_cast<int64_t*>(dctr + 2 * nchunks);    // [chunk][begin, end]
  int64_t* dtotal = drange + 2 * nchunks;                               // running dense total
  long long* dtile = reinterpret_cast<long long*>(dtotal + 1);           // scan tile sums
  int64_t* hinfo = h->hinfo;                                            // [chunk][begin, end, retry, -]
  h->last_kernel_ms = 0.0;
  // Cost ordering within each chunk (lean batches of short pairs).
  const bool order = orders_batch(h, b);
  OrderBufs ob{};
  if (order) {
    if (int e = order_bufs(h, n, nchunks, &ob)) return e;
    if (cudaMemsetAsync(ob.hist, 0, (size_t)nchunks * kOrderStride * 4, sc) != cudaSuccess)
      return fail(h, WFA_ERR_CUDA, "memset");
  }

#define PIPE_TRY(expr, what)                                                                      \
  do {                                                                                            \
    cudaError_t _e = (expr);                                                                      \
    if (_e != cudaSuccess)                                                                        \
      return fail(h, _e == cudaErrorMemoryAllocation ? WFA_ERR_OOM : WFA_ERR_CUDA, what, _e);     \
  } while (0)

  if (aln) PIPE_TRY(cudaMemsetAsync(dtotal, 0, 8, sc), "memset");
  // Every chunk: inputs in (s_in); slot offsets, the alignment, the dense
  // CIGAR offsets and the compaction (compute stream, a few short launches
  // around the alignment kernel); results, chunk info and CIGAR bytes out
  // (s_out) while the next chunk aligns.
  for (int64_t ci = 0; ci < nchunks; ++ci) {
    const int64_t a = bnd[(size_t)ci], e = bnd[(size_t)ci + 1], cn = e - a;
    const ChunkInfo& I = ci_info[(size_t)ci];
    if (I.hi > I.lo)
      PIPE_TRY(cudaMemcpyAsync(dseq + I.lo, (const uint8_t*)b->seq + I.lo, (size_t)(I.hi - I.lo),
                               cudaMemcpyHostToDevice, si), "H2D");
    PIPE_TRY(cudaMemcpyAsync(dpo + a, b->p_off + a, (size_t)cn * 8, cudaMemcpyHostToDevice, si), "H2D");
    PIPE_TRY(cudaMemcpyAsync(dto + a, b->t_off + a, (size_t)cn * 8, cudaMemcpyHostToDevice, si), "H2D");
    PIPE_TRY(cudaMemcpyAsync(dpl + a, b->p_len + a, (size_t)cn * 4, cudaMemcpyHostToDevice, si), "H2D");
    PIPE_TRY(cudaMemcpyAsync(dtl + a, b->t_len + a, (size_t)cn * 4, cudaMemcpyHostToDevice, si), "H2D");
    PIPE_TRY(cudaEventRecord(ev_in[(size_t)ci], si), "event");
    PIPE_TRY(cudaStreamWaitEvent(sc, ev_in[(size_t)ci], 0), "wait");
    if (aln) {
      PIPE_TRY(chunk_scan<0>(dpl + a, dtl + a, nullptr, cn, c_slot0[(size_t)ci], nullptr, dco + a, nullptr,
                             dtile, sc), "slot offsets");
      h->launches += 3;
    }
    wfa_batch_t cb = *b;
    cb.num_pairs = cn;
    cb.seq = dseq;
    cb.seq_bytes = (int64_t)seq_bytes;
    cb.p_off = dpo + a; cb.t_off = dto + a; cb.p_len = dpl + a; cb.t_len = dtl + a;
    cb.cigar_off = aln ? dco + a : nullptr;
    cb.cigar_bytes = slot_total;
    AlignParams P;
    fill_params(h, &cb, P);
    P.results = dres + a;
    P.cigars = aln ? h->cigars.as<uint8_t>() : nullptr;
    // Lanes per pair: the tuned choice of a device batch of this kind, if
    // one ran in this process, else the bucket's default (chunks are not
    // timed here: the pipeline would wait on them).
    const int lanes = choose_lanes(h, P, I.max_len_sum, cn, sc, false);
    Round rd = first_round(P, metric_components(P.metric), I.max_len_sum, lanes, true, I.max_seq);
    const int64_t* clist = nullptr;
    if (order && cn >= kSortMinPairs && length_bucket(I.max_len_sum) <= 2) {
      int32_t* hst = ob.hist + kOrderStride * ci;
      int32_t* dmx = hst + 2 * kOrderBins;  // the chunk's longest pair (known here already)
      int nl = 0;
      PIPE_TRY(launch_order(dseq, packed, dpo + a, dpl + a, dto + a, dtl + a, cn, h->num_sms, dmx, ob.keys + a,
                            hst, hst + kOrderBins, ob.list + a, sc, &nl),
               "cost order");
      h->launches += nl;
      clist = ob.list + a;
    }
    PIPE_TRY(cudaEventRecord(h->evtime[2 * (size_t)ci], sc), "event");
    int e2 = launch_round(h, P, rd, cn, clist, sc, dctr + 2 * ci);
    if (e2 != WFA_OK) return e2;
    PIPE_TRY(cudaEventRecord(h->evtime[2 * (size_t)ci + 1], sc), "event");
    if (ci == 0) h->last_lanes = h->launch_lanes;
    PIPE_TRY(cudaEventRecord(ev_k[(size_t)ci], sc), "event");
    cudaEvent_t ready = ev_k[(size_t)ci];
    if (aln) {
      PIPE_TRY(chunk_scan<1>(nullptr, nullptr, dres + a, cn, 0, dtotal, ddst + a, drange + 2 * ci, dtile,
                             sc), "dense offsets");
      compact_cigars<<<(unsigned)((cn * 32 + 255) / 256), 256, 0, sc>>>(
          dres + a, dco + a, h->cigars.as<uint8_t>(), ddst + a, h->dense.as<uint8_t>(), cn);
      h->launches += 4;
      PIPE_TRY(cudaGetLastError(), "compact cigars");
      PIPE_TRY(cudaEventRecord(ev_x[(size_t)ci], sc), "event");
      ready = ev_x[(size_t)ci];
    }
    PIPE_TRY(cudaStreamWaitEvent(so, ready, 0), "wait");
    PIPE_TRY(cudaMemcpyAsync(results + a, dres + a, (size_t)cn * sizeof(wfa_result_t), cudaMemcpyDeviceToHost, so), "D2H");
    if (aln)
      PIPE_TRY(cudaMemcpyAsync(hinfo + 4 * ci, drange + 2 * ci, 16, cudaMemcpyDeviceToHost, so), "D2H");
    PIPE_TRY(cudaMemcpyAsync(hinfo + 4 * ci + 2, dctr + 2 * ci + 1, 8, cudaMemcpyDeviceToHost, so), "D2H");
    PIPE_TRY(cudaEventRecord(ev_res[(size_t)ci], so), "event");
  }

  // As each chunk's info arrives: its dense CIGAR bytes out, on their own
  // stream (s_out already holds every later chunk's result copies).
  std::vector<int64_t> retry;
  int64_t dense_total = 0;
  for (int64_t ci = 0; ci < nchunks; ++ci) {
    const int64_t a = bnd[(size_t)ci], e = bnd[(size_t)ci + 1];
    PIPE_TRY(cudaEventSynchronize(ev_res[(size_t)ci]), "results");
    const int32_t nretry = (int32_t)(hinfo[4 * ci + 2] & 0xffffffff);
    if (nretry > 0)
      for (int64_t i = a; i < e; ++i)
        if (results[i].status == kStatusRetry) { retry.push_back(i); results[i].cigar_length = 0; }
    if (!aln) continue;
    const int64_t d0 = hinfo[4 * ci], d1 = hinfo[4 * ci + 1];
    if (d1 > d0)
      PIPE_TRY(cudaMemcpyAsync(cigars + d0, h->dense.as<uint8_t>() + d0, (size_t)(d1 - d0),
                               cudaMemcpyDeviceToHost, h->s_cig), "D2H");
    dense_total = d1;
  }
  PIPE_TRY(cudaStreamSynchronize(so), "D2H");
  PIPE_TRY(cudaStreamSynchronize(h->s_cig), "D2H");
  PIPE_TRY(cudaStreamSynchronize(sc), "compute");
  for (int64_t ci = 0; ci < nchunks; ++ci) {
    float ms = 0.f;
    PIPE_TRY(cudaEventElapsedTime(&ms, h->evtime[2 * (size_t)ci], h->evtime[2 * (size_t)ci + 1]), "event");
    h->last_kernel_ms += ms;
  }
#undef PIPE_TRY


  // Pairs that outgrew the first configuration: re-run with the batch driver.
  if (!retry.empty()) {
    const int64_t rn = (int64_t)retry.size();
    h->last_reruns += rn;
    std::vector<int64_t> po(rn), to(rn), co(rn);
    std::vector<int32_t> pl(rn), tl(rn);
    int32_t mx = 0;
    int64_t rslot = 0;
    for (int64_t j = 0; j < rn; ++j) {
      int64_t i = retry[(size_t)j];
      po[j] = b->p_off[i]; to[j] = b->t_off[i]; pl[j] = b->p_len[i]; tl[j] = b->t_len[i];
      mx = std::max<int32_t>(mx, pl[j] + tl[j]);
      co[j] = rslot;
      rslot += 2 * ((int64_t)pl[j] + tl[j]) + 1;
    }
    DevBuf rbuf;
    rbuf.st = sc;
    size_t need = (size_t)rn * (8 * 3 + 4 * 2 + sizeof(wfa_result_t)) + (size_t)rslot + 64;
    CUDA_TRY(h, rbuf.ensure(need), "retry buffers");
    char* base = rbuf.as<char>();
    int64_t* rpo = reinterpret_cast<int64_t*>(base);
    int64_t* rto = rpo + rn;
    int64_t* rco = rto + rn;
    int32_t* rpl = reinterpret_cast<int32_t*>(rco + rn);
    int32_t* rtl = rpl + rn;
    wfa_result_t* rres = reinterpret_cast<wfa_result_t*>(reinterpret_cast<char*>(rtl + rn) + ((rn & 1) ? 4 : 0));
    uint8_t* rcig = reinterpret_cast<uint8_t*>(rres + rn);
    cudaMemcpyAsync(rpo, po.data(), rn * 8, cudaMemcpyHostToDevice, sc);
    cudaMemcpyAsync(rto, to.data(), rn * 8, cudaMemcpyHostToDevice, sc);
    cudaMemcpyAsync(rco, co.data(), rn * 8, cudaMemcpyHostToDevice, sc);
    cudaMemcpyAsync(rpl, pl.data(), rn * 4, cudaMemcpyHostToDevice, sc);
    cudaMemcpyAsync(rtl, tl.data(), rn * 4, cudaMemcpyHostToDevice, sc);
    wfa_batch_t rb = *b;
    rb.num_pairs = rn;
    rb.seq = dseq;
    rb.seq_bytes = (int64_t)seq_bytes;
    rb.p_off = rpo; rb.t_off = rto; rb.p_len = rpl; rb.t_len = rtl;
    rb.cigar_off = aln ? rco : nullptr;
    rb.cigar_bytes = rslot;
    double kms = h->last_kernel_ms;
    int e3 = run_device_batch(h, &rb, rres, aln ? rcig : nullptr, sc, mx);
    h->last_kernel_ms += kms;
    if (e3 != WFA_OK) { rbuf.release(); return e3; }
    std::vector<wfa_result_t> rr((size_t)rn);
    std::vector<uint8_t> rc(aln ? (size_t)rslot : 0);
    cudaMemcpyAsync(rr.data(), rres, rn * sizeof(wfa_result_t), cudaMemcpyDeviceToHost, sc);
    if (aln) cudaMemcpyAsync(rc.data(), rcig, (size_t)rslot, cudaMemcpyDeviceToHost, sc);
    cudaError_t es = cudaStreamSynchronize(sc);
    rbuf.release();
    if (es != cudaSuccess) return fail(h, WFA_ERR_CUDA, "retry D2H", es);
    for (int64_t j = 0; j < rn; ++j) {
      int64_t i = retry[(size_t)j];
      wfa_result_t x = rr[(size_t)j];
      if (aln && x.cigar_length > 0) {
        std::memcpy(cigars + dense_total, rc.data() + co[j] + x.cigar_begin, (size_t)x.cigar_length);
        x.cigar_begin = (int32_t)dense_total;
        dense_total += x.cigar_length;
      } else {
        x.cigar_begin = 0;
      }
      results[i] = x;
    }
  }
  return WFA_OK;
}

static void async_loop(wfa_aligner_t* h) {
  cudaSetDevice(h->device);
  for (;;) {
    wfa_aligner_t::Job job;
    {
      std::unique_lock<std::mutex> lock(h->async_mu);
      h->async_cv.wait(lock, [&] { return h->async_stop || !h->async_jobs.empty(); });
      if (h->async_jobs.empty()) return;
      job = h->async_jobs.front();
      h->async_jobs.pop_front();
    }
    const int rc = wfa_batch_align(h, &job.batch, job.results, job.cigars);
    {
      std::lock_guard<std::mutex> lock(h->async_mu);
      h->async_done[job.ticket] = rc;
    }
    h->async_cv.notify_all();
  }
}

int64_t wfa_batch_submit(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results,
                         uint8_t* cigars) {
  if (!h || !b || !results) return WFA_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(h->async_mu);
  if (h->async_stop) return WFA_ERR_ARGUMENT;
  if (!h->async_worker.joinable()) h->async_worker = std::thread(async_loop, h);
  const int64_t t = h->async_next++;
  h->async_jobs.push_back(wfa_aligner_t::Job{t, *b, results, cigars});
  h->async_cv.notify_all();
  return t;
}

int wfa_batch_poll(wfa_aligner_t* h, int64_t ticket, int* status) {
  if (!h || ticket < 0) return WFA_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(h->async_mu);
  auto it = h->async_done.find(ticket);
  if (it == h->async_done.end()) return ticket < h->async_next ? 0 : WFA_ERR_ARGUMENT;
  if (status) *status = it->second;
  h->async_done.erase(it);
  return 1;
}

int wfa_batch_wait(wfa_aligner_t* h, int64_t ticket) {
  if (!h || ticket < 0) return WFA_ERR_ARGUMENT;
  std::unique_lock<std::mutex> lock(h->async_mu);
  if (ticket >= h->async_next) return WFA_ERR_ARGUMENT;
  h->async_cv.wait(lock, [&] { return h->async_done.count(ticket) > 0; });
  const int rc = h->async_done[ticket];
  h->async_done.erase(ticket);
  return rc;
}

int32_t wfa_cigar_rle(const uint8_t* ops, int32_t len, char* out, int32_t cap) {
  std::string r;
  int32_t i = 0;
  char tmp[24];
  while (i < len) {
    int32_t j = i;
    while (j < len && ops[j] == ops[i]) ++j;
    std::snprintf(tmp, sizeof tmp, "%d%c", j - i, ops[i]);
    r += tmp;
    i = j;
  }
  if (out && cap > 0) {
    int32_t c = std::min<int32_t>((int32_t)r.size(), cap - 1);
    std::memcpy(out, r.data(), (size_t)c);
    out[c] = 0;
  }
  return (int32_t)r.size();
}

const char* wfa_version(void) { return "wfa2lib-rs_b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace wfab {
cudaError_t preload_order_kernels();

// Loads every kernel of the library on `device` now.  CUDA loads a kernel
// at its first launch, and loading waits until the kernels already running
// on the device have finished: beside a resident stream's kernel (which
// runs until it has been idle for about a second) a batch lane's first
// launch of each kernel would wait that long.  The occupancy queries load
// their kernel (cudaFuncGetAttributes), so one query per instantiation
// loads them all.
int preload_kernels(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return WFA_ERR_CUDA;
  cudaFuncAttributes a;
  for (const void* f : {(const void*)collect_retries, (const void*)compact_cigars, (const void*)scan_tiles<0, false>,
                        (const void*)scan_tiles<0, true>, (const void*)scan_tiles<1, false>,
                        (const void*)scan_tiles<1, true>, (const void*)scan_tile_offsets, (const void*)max_lengths,
                        (const void*)collect_retries_capped})
    if (cudaFuncGetAttributes(&a, f) != cudaSuccess) return WFA_ERR_CUDA;
  if (preload_order_kernels() != cudaSuccess) return WFA_ERR_CUDA;
  for (int metric : {(int)WFA_METRIC_EDIT, (int)WFA_METRIC_GAP_LINEAR, (int)WFA_METRIC_GAP_AFFINE,
                     (int)WFA_METRIC_GAP_AFFINE_2P}) {
    const int cls = metric_class(metric);
    AlignParams P{};
    P.metric = metric;
    P.compute_alignment = 1;
    for (int fmt : {(int)WFA_SEQ_ASCII, (int)WFA_SEQ_PACKED2}) {
      P.format = fmt;
      P.span = WFA_SPAN_END2END;
      P.piggyback = 0;
      P.hkind = WFA_HEURISTIC_NONE;
      for (int lanes : {4, 8, 16, 32}) occupancy_blocks_per_sm(P, cls, lanes, 0);
      for (int lanes : {32, 128, 256, 512}) occupancy_biwfa(P, cls, lanes, 0);
      P.hkind = WFA_HEURISTIC_WFADAPTIVE;  // the kernels with heuristic support
      occupancy_blocks_per_sm(P, cls, 32, 0);
      occupancy_biwfa(P, cls, 32, 0);
      P.hkind = WFA_HEURISTIC_NONE;
      P.piggyback = 1;  // med/low
      occupancy_blocks_per_sm(P, cls, 32, 0);
    }
    for (int lanes : {8, 32}) occupancy_resident(cls, lanes, 0);
  }
  cudaGetLastError();
  return WFA_OK;
}
}  // namespace wfab

// ---------------------------------------------------------------------------
// Resident stream (wfa_stream_*): a persistent kernel (wfa_resident.cu) fed
// from a request ring in mapped host memory.  Host side: the ring and its
// slots' bookkeeping, the kernel's launches and relaunches, the results.
// ---------------------------------------------------------------------------
namespace {

using StreamClock = std::chrono::steady_clock;

template <class T>
T* host_mapped(size_t count, T** dev) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, std::max<size_t>(count * sizeof(T), 64), cudaHostAllocMapped) != cudaSuccess) return nullptr;
  std::memset(p, 0, std::max<size_t>(count * sizeof(T), 64));
  void* d = nullptr;
  if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
    cudaFreeHost(p);
    return nullptr;
  }
  *dev = reinterpret_cast<T*>(d);
  return reinterpret_cast<T*>(p);
}

// Polls of the doorbell (about 1.5 us each) without a new request before a
// launch ends, and a lane group's polls (backing off to about 8 us) before it
// gives up.
constexpr int64_t kStreamIdlePolls = 700000;
constexpr int64_t kStreamGroupPolls = 4000000;

}  // namespace

struct wfa_stream {
  wfa_aligner_t* h = nullptr;   // the kernel's handle: its stream and scratch
  wfa_aligner_t* fb = nullptr;  // requests that outgrow the kernel's scratch (made on first need)
  int metric = 0;
  wfa_penalties_t pen{};
  int score_only = 0;
  // Mapped host memory (host views; the device views are in R).
  ResidentCtl* ctl = nullptr;
  ResidentReq* reqs = nullptr;
  uint8_t* arena = nullptr;
  wfa_result_t* results = nullptr;
  uint8_t* cigars = nullptr;
  uint32_t* done = nullptr;
  unsigned long long* xfer = nullptr;  // pinned words for the device counters
  DevBuf dev;                          // head, dtail, dstop
  ResidentArgs R{};
  AlignParams P{};
  int cls = 0, lanes = 32, blocks = 0;
  size_t smem = 0;
  int64_t cap = 0;
  int32_t max_len_sum = 0;
  std::mutex mu;
  uint64_t tail = 0, oldest = 0;
  uint64_t served = 0;  // requests below this were served by ended launches
  std::vector<int64_t> t_submit;  // per slot (steady clock ns)
  std::vector<uint8_t> taken;     // per slot: its result was returned
  bool running = false;
  cudaEvent_t ended = nullptr;
  int64_t launches = 0, fallbacks = 0;
  std::string err;
};

namespace {

void stream_free(wfa_stream_t* s) {
  if (s->ended) cudaEventDestroy(s->ended);
  for (void* p : {(void*)s->ctl, (void*)s->reqs, (void*)s->arena, (void*)s->results, (void*)s->cigars,
                  (void*)s->done, (void*)s->xfer})
    if (p) cudaFreeHost(p);
  s->dev.release();
  if (s->h) wfa_aligner_destroy(s->h);
  if (s->fb) wfa_aligner_destroy(s->fb);
  delete s;
}

// Launches the kernel over what is published (caller holds mu): tickets
// start at the first request no launch served (`served`), the mirrored tail
// at what is published.
int stream_launch(wfa_stream_t* s) {
  wfa_aligner_t* h = s->h;
  s->xfer[0] = s->served;
  s->xfer[1] = s->tail;
  CUDA_TRY(h, cudaMemcpyAsync(s->R.head, s->xfer, 16, cudaMemcpyHostToDevice, h->stream), "stream counters");
  CUDA_TRY(h, cudaMemsetAsync(s->R.dstop, 0, 4, h->stream), "stream stop flag");
  CUDA_TRY(h, cudaGetLastError(), "an earlier CUDA call of this thread");
  CUDA_TRY(h, launch_resident(s->P, s->R, s->cls, s->lanes, s->blocks, s->smem, h->stream),
           "resident kernel launch");
  CUDA_TRY(h, cudaEventRecord(s->ended, h->stream), "event");
  s->running = true;
  ++s->launches;
  ++h->launches;
  return WFA_OK;
}

// Notices the end of a launch; relaunches when requests were published that
// no launch claimed (caller holds mu).
int stream_tend(wfa_stream_t* s) {
  if (!s->err.empty()) return WFA_ERR_CUDA;
  wfa_aligner_t* h = s->h;
  if (s->running) {
    const cudaError_t q = cudaEventQuery(s->ended);
    if (q == cudaErrorNotReady) return WFA_OK;
    if (q != cudaSuccess) {
      s->err = std::string("resident kernel: ") + cudaGetErrorString(q);
      s->running = false;
      return WFA_ERR_CUDA;
    }
    s->running = false;
  }
  if (s->tail == s->served) return WFA_OK;
  if (s->launches > 0) {
    // The launch that ended served every request below the tail it saw last.
    CUDA_TRY(h, cudaMemcpyAsync(s->xfer, s->R.dtail, 8, cudaMemcpyDeviceToHost, h->stream), "stream tail");
    CUDA_TRY(h, cudaStreamSynchronize(h->stream), "stream tail");
    if (s->ctl->gave_up > 0) {
      s->err = "resident kernel: a lane group gave up waiting for its request";
      return WFA_ERR_CUDA;
    }
    s->served = s->xfer[0];
  }
  if (s->served < s->tail) return stream_launch(s);
  return WFA_OK;
}

void publish(wfa_stream_t* s) {
  std::atomic_thread_fence(std::memory_order_release);
  *reinterpret_cast<volatile unsigned long long*>(&s->ctl->tail) = s->tail;
}

int64_t stream_put(wfa_stream_t* s, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m,
                   int64_t now) {
  const int64_t i = (int64_t)(s->tail % (uint64_t)s->cap);
  s->reqs[i] = ResidentReq{n, m};
  uint8_t* a = s->arena + i * s->R.seq_stride;
  if (n) std::memcpy(a, p, (size_t)n);
  if (m) std::memcpy(a + n, t, (size_t)m);
  s->t_submit[(size_t)i] = now;
  s->taken[(size_t)i] = 0;
  return (int64_t)s->tail++;
}

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(StreamClock::now().time_since_epoch()).count();
}

// The result of slot i through the host-buffer batch path (a request whose
// alignment outgrew the kernel's scratch).
int stream_fallback(wfa_stream_t* s, int64_t i, wfa_result_t* r, std::vector<uint8_t>* cig) {
  if (!s->fb) {
    int e = WFA_OK;
    s->fb = wfa_aligner_create((wfa_metric_t)s->metric, &s->pen, s->h->device, &e);
    if (!s->fb) return e;
    wfa_set_alignment_scope(s->fb, s->score_only ? WFA_SCOPE_SCORE : WFA_SCOPE_ALIGNMENT);
  }
  const ResidentReq q = s->reqs[i];
  const int64_t po = 0, to = q.n;
  const int32_t pl = q.n, tl = q.m;
  wfa_batch_t b{};
  b.format = WFA_SEQ_ASCII;
  b.span = WFA_SPAN_END2END;
  b.num_pairs = 1;
  b.seq = s->arena + i * s->R.seq_stride;
  b.seq_bytes = (int64_t)q.n + q.m;
  b.p_off = &po;
  b.p_len = &pl;
  b.t_off = &to;
  b.t_len = &tl;
  cig->assign(2 * ((size_t)q.n + q.m) + 16, 0);
  ++s->fallbacks;
  return wfa_batch_align(s->fb, &b, r, s->score_only ? nullptr : cig->data());
}

}  // namespace

extern "C" {

wfa_stream_t* wfa_stream_start(wfa_metric_t metric, const wfa_penalties_t* penalties, int32_t device,
                               int32_t score_only, int32_t max_len_sum, int32_t capacity,
                               int32_t blocks_per_sm, int* err) {
  auto bad = [&](int e) -> wfa_stream_t* {
    if (err) *err = e;
    return nullptr;
  };
  if (max_len_sum < 1 || max_len_sum > kLongPair || capacity < 1 || blocks_per_sm < 0)
    return bad(WFA_ERR_ARGUMENT);
  int e = WFA_OK;
  wfa_aligner_t* h = wfa_aligner_create(metric, penalties, device, &e);
  if (!h) return bad(e);
  wfa_stream_t* s = new wfa_stream();
  s->h = h;
  s->metric = metric;
  if (penalties) s->pen = *penalties;
  s->score_only = score_only ? 1 : 0;
  s->cap = capacity;
  s->max_len_sum = max_len_sum;
  wfa_set_alignment_scope(h, score_only ? WFA_SCOPE_SCORE : WFA_SCOPE_ALIGNMENT);
  // Launch shape: the first round of a host batch of such pairs.
  wfa_batch_t b{};
  b.format = WFA_SEQ_ASCII;
  b.span = WFA_SPAN_END2END;
  fill_params(h, &b, s->P);
  s->cls = metric_class(s->P.metric);
  const int nc = metric_components(s->P.metric);
  s->lanes = max_len_sum <= 512 ? 8 : 32;
  Round r = first_round(s->P, nc, max_len_sum, s->lanes, true, max_len_sum);
  int64_t group_words = 0;
  SmemLayout L = round_layout(s->P, r, nc, &group_words);
  if (L.total > 200 * 1024 && s->lanes == 8) {
    s->lanes = 32;
    r = first_round(s->P, nc, max_len_sum, s->lanes, true, max_len_sum);
    L = round_layout(s->P, r, nc, &group_words);
  }
  if (L.total > 200 * 1024) {
    stream_free(s);
    return bad(WFA_ERR_UNSUPPORTED);
  }
  s->smem = L.total;
  const int64_t seq_stride = ((int64_t)max_len_sum + 16 + 15) & ~(int64_t)15;
  const int64_t cig_stride = (2 * (int64_t)max_len_sum + 1 + 15) & ~(int64_t)15;
  // After the ring and history (aligned to 16 bytes): the request's bytes
  // and its CIGAR.
  group_words = ((group_words + 4 + (seq_stride + cig_stride) / 4) + 63) & ~(int64_t)63;
  int occ = occupancy_resident(s->cls, s->lanes, s->smem);
  if (blocks_per_sm > 0) occ = std::min(occ, (int)blocks_per_sm);
  s->blocks = h->num_sms * std::max(1, occ);
  const int gpb = kWarpsPerBlock * 32 / s->lanes;
  s->dev.st = h->stream;
  bool ok = h->scratch.ensure((size_t)s->blocks * gpb * group_words * 4) == cudaSuccess &&
            s->dev.ensure(64) == cudaSuccess;
  ok = ok && cudaMemsetAsync(s->dev.p, 0, 64, h->stream) == cudaSuccess &&
       cudaStreamSynchronize(h->stream) == cudaSuccess && cudaEventCreate(&s->ended) == cudaSuccess;
  ResidentArgs& R = s->R;
  ResidentCtl* ctl_d = nullptr;
  ResidentReq* reqs_d = nullptr;
  uint8_t *arena_d = nullptr, *cig_d = nullptr;
  wfa_result_t* res_d = nullptr;
  uint32_t* done_d = nullptr;
  unsigned long long* xfer_d = nullptr;
  ok = ok && (s->ctl = host_mapped<ResidentCtl>(1, &ctl_d)) && (s->reqs = host_mapped<ResidentReq>((size_t)s->cap, &reqs_d)) &&
       (s->arena = host_mapped<uint8_t>((size_t)(s->cap * seq_stride), &arena_d)) &&
       (s->results = host_mapped<wfa_result_t>((size_t)s->cap, &res_d)) &&
       (s->cigars = host_mapped<uint8_t>((size_t)(s->cap * cig_stride), &cig_d)) &&
       (s->done = host_mapped<uint32_t>((size_t)s->cap, &done_d)) &&
       (s->xfer = host_mapped<unsigned long long>(2, &xfer_d));
  if (!ok) {
    cudaGetLastError();
    stream_free(s);
    return bad(WFA_ERR_OOM);
  }
  s->P.scratch = h->scratch.as<int32_t>();
  s->P.warp_words = group_words;
  R.ctl = ctl_d;
  R.reqs = reqs_d;
  R.arena = arena_d;
  R.results = res_d;
  R.cigars = cig_d;
  R.done = done_d;
  R.cap = s->cap;
  R.seq_stride = seq_stride;
  R.cig_stride = cig_stride;
  unsigned long long* d = s->dev.as<unsigned long long>();
  R.head = d;
  R.dtail = d + 1;
  R.dstop = reinterpret_cast<int32_t*>(d + 2);
  R.idle_polls = kStreamIdlePolls;
  R.group_polls = kStreamGroupPolls;
  s->t_submit.assign((size_t)s->cap, 0);
  s->taken.assign((size_t)s->cap, 0);
  if (err) *err = WFA_OK;
  return s;
}

int64_t wfa_stream_submit(wfa_stream_t* s, const uint8_t* pattern, int32_t n, const uint8_t* text, int32_t m) {
  if (!s || n < 0 || m < 0 || (n > 0 && !pattern) || (m > 0 && !text) || (int64_t)n + m > s->max_len_sum)
    return WFA_ERR_ARGUMENT;
  const int64_t now = now_ns();
  std::lock_guard<std::mutex> lock(s->mu);
  if (!s->err.empty()) return WFA_ERR_CUDA;
  if ((int64_t)(s->tail - s->oldest) >= s->cap) return WFA_ERR_BUSY;
  const int64_t id = stream_put(s, pattern, n, text, m, now);
  publish(s);
  const int rc = stream_tend(s);
  return rc == WFA_OK ? id : rc;
}

int64_t wfa_stream_submit_many(wfa_stream_t* s, const uint8_t* seq, const int64_t* p_off, const int32_t* p_len,
                               const int64_t* t_off, const int32_t* t_len, int64_t count) {
  if (!s || count < 0 || (count > 0 && (!seq || !p_off || !p_len || !t_off || !t_len))) return WFA_ERR_ARGUMENT;
  for (int64_t j = 0; j < count; ++j)
    if (p_len[j] < 0 || t_len[j] < 0 || (int64_t)p_len[j] + t_len[j] > s->max_len_sum) return WFA_ERR_ARGUMENT;
  const int64_t now = now_ns();
  std::lock_guard<std::mutex> lock(s->mu);
  if (!s->err.empty()) return WFA_ERR_CUDA;
  if ((int64_t)(s->tail - s->oldest) + count > s->cap) return WFA_ERR_BUSY;
  const int64_t first = (int64_t)s->tail;
  for (int64_t j = 0; j < count; ++j) stream_put(s, seq + p_off[j], p_len[j], seq + t_off[j], t_len[j], now);
  publish(s);
  const int rc = stream_tend(s);
  return rc == WFA_OK ? first : rc;
}

int32_t wfa_stream_poll(wfa_stream_t* s, wfa_served_t* out, int32_t max, uint8_t* cigars, int64_t cigar_cap,
                        int32_t timeout_ms) {
  if (!s || !out || max <= 0) return WFA_ERR_ARGUMENT;
  const auto deadline = StreamClock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
  std::vector<uint8_t> fcig;
  for (;;) {
    {
      std::lock_guard<std::mutex> lock(s->mu);
      if (!s->err.empty()) return WFA_ERR_CUDA;
      int32_t c = 0;
      int64_t used = 0;
      for (uint64_t q = s->oldest; q < s->tail && c < max; ++q) {
        const int64_t i = (int64_t)(q % (uint64_t)s->cap);
        if (s->taken[(size_t)i]) continue;
        const uint32_t mark = *reinterpret_cast<volatile uint32_t*>(s->done + i);
        if (mark != (uint32_t)(q / (uint64_t)s->cap) + 1u) continue;
        std::atomic_thread_fence(std::memory_order_acquire);
        const int64_t t_done = now_ns();
        wfa_result_t r = s->results[i];
        const uint8_t* ops = s->cigars + i * s->R.cig_stride;
        if (r.status == kStatusRetry) {
          const int rc = stream_fallback(s, i, &r, &fcig);
          if (rc != WFA_OK) {
            r.status = rc;
            r.score = 0;
            r.cigar_length = 0;
          }
          ops = fcig.data() + r.cigar_begin;
        }
        const int64_t len = s->score_only ? 0 : r.cigar_length;
        wfa_served_t& o = out[c];
        std::memset(&o, 0, sizeof o);
        o.cigar_offset = -1;
        if (len > 0) {
          if (!cigars || used + len > cigar_cap) {
            if (c == 0) return WFA_ERR_ARGUMENT;  // the next CIGAR does not fit the buffer
            break;
          }
          std::memcpy(cigars + used, ops, (size_t)len);
          o.cigar_offset = used;
          used += len;
        }
        o.id = (int64_t)q;
        o.score = r.score;
        o.status = r.status;
        o.cigar_length = (int32_t)len;
        o.cigar_score = r.cigar_score;
        o.end_v = r.end_v;
        o.end_h = r.end_h;
        o.mode = 0;
        o.latency_ns = t_done - s->t_submit[(size_t)i];
        s->taken[(size_t)i] = 1;
        ++c;
      }
      while (s->oldest < s->tail && s->taken[(size_t)(s->oldest % (uint64_t)s->cap)]) {
        s->taken[(size_t)(s->oldest % (uint64_t)s->cap)] = 0;
        ++s->oldest;
      }
      if (c > 0) return c;
      const int rc = stream_tend(s);
      if (rc != WFA_OK) return rc;
    }
    if (StreamClock::now() >= deadline) return 0;
    std::this_thread::sleep_for(std::chrono::microseconds(10));
  }
}

int64_t wfa_stream_pending(wfa_stream_t* s) {
  if (!s) return WFA_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  return (int64_t)(s->tail - s->oldest);
}

int wfa_stream_stats(wfa_stream_t* s, int64_t* out, int32_t n) {
  if (!s || !out || n < 0) return WFA_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  const int64_t v[6] = {s->launches, (int64_t)s->ctl->idle_exits, (int64_t)s->ctl->gave_up, s->fallbacks,
                        s->blocks, s->lanes};
  for (int32_t j = 0; j < n && j < 6; ++j) out[j] = v[j];
  return WFA_OK;
}

int wfa_stream_stop(wfa_stream_t* s) {
  if (!s) return WFA_ERR_ARGUMENT;
  int rc = WFA_OK;
  {
    // With stop set, a running launch (or one started here for requests no
    // launch claimed) aligns what was published and returns.
    std::lock_guard<std::mutex> lock(s->mu);
    *reinterpret_cast<volatile int32_t*>(&s->ctl->stop) = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    rc = stream_tend(s);
  }
  if (cudaStreamSynchronize(s->h->stream) != cudaSuccess) rc = WFA_ERR_CUDA;
  stream_free(s);
  return rc;
}

}  // extern "C"
