// wfa_capi.cu -- host side of the C ABI (include/wfa_b200.h).
//
// A handle mirrors one reference WavefrontAligner (src/aligner.rs:146): its
// builder state, the last alignment's status and CIGAR, and the device
// resources it reuses across calls (input/output buffers, per-warp scratch,
// a stream).  Alignments always run on the GPU: there is no CPU path, and a
// configuration this build cannot run on the device is refused with
// WFA_ERR_UNSUPPORTED.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "wfa_common.h"
#include "wfa_kernels.h"
#include "wfa_params.h"

using namespace wfab;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

struct ScratchCfg {
  int32_t wmax;
  int32_t hist_scores;
  int64_t hist_words;
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
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  DevBuf seq, poff, plen, toff, tlen, coff, results, cigars, dense, scratch, counters, pairlist;
  int64_t launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_kernel_ms = 0.0;
};

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
// per pair, coalesced byte copies).
__global__ void compact_cigars(const wfa_result_t* res, const int64_t* slot_off,
                               const uint8_t* slots, const int64_t* dst_off, uint8_t* dense,
                               int64_t n) {
  int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= n) return;
  int32_t len = res[w].cigar_length;
  const uint8_t* src = slots + slot_off[w] + res[w].cigar_begin;
  uint8_t* dst = dense + dst_off[w];
  for (int32_t i = lane; i < len; i += 32) dst[i] = src[i];
}

__global__ void max_lengths(const int32_t* pl, const int32_t* tl, int64_t n, int32_t* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t v = 0;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) v = max(v, pl[i] + tl[i]);
  v = __reduce_max_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) atomicMax(out, v);
}

// ---------------------------------------------------------------------------
// Configuration checks
// ---------------------------------------------------------------------------
static int check_supported(wfa_aligner_t* h, bool biwfa) {
  if (biwfa) return fail(h, WFA_ERR_UNSUPPORTED, "BiWFA is not available in this build");
  if (h->scope == WFA_SCOPE_ALIGNMENT && h->memory_mode != WFA_MEMORY_HIGH)
    return fail(h, WFA_ERR_UNSUPPORTED,
                "med/low memory (piggyback backtrace) is not available in this build");
  if (h->compat == WFA_COMPAT_CORRECTED && h->pen.match < 0 && h->span == WFA_SPAN_ENDSFREE)
    return fail(h, WFA_ERR_UNSUPPORTED, "Compat::Corrected ends-free with a match reward");
  if (h->pen.scope > 1024) return fail(h, WFA_ERR_UNSUPPORTED, "max_score_scope above 1024");
  return WFA_OK;
}

static void fill_params(const wfa_aligner_t* h, const wfa_batch_t* b, AlignParams& P) {
  P = h->pen;
  P.span = b->span;
  P.extension = b->span == WFA_SPAN_ENDSFREE ? h->extension : 0;
  P.p0 = h->p0; P.pf = h->pf; P.t0 = h->t0; P.tf = h->tf;
  P.hkind = h->hkind; P.hp0 = h->hp0; P.hp1 = h->hp1; P.hp2 = h->hp2;
  P.compute_alignment = h->scope == WFA_SCOPE_ALIGNMENT;
  P.max_steps = h->max_steps;
  P.format = b->format;
  P.seq = static_cast<const uint8_t*>(b->seq);
  P.seq_bytes = b->seq_bytes;
  P.p_off = b->p_off; P.p_len = b->p_len; P.t_off = b->t_off; P.t_len = b->t_len;
  P.cigar_off = b->cigar_off;
  P.num_pairs = b->num_pairs;
  P.pair_list = nullptr;
}

// Runs every pair of a device-resident batch, escalating scratch for pairs
// that need more.  Synchronises `st` to read the retry count.
static int run_device_batch(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* d_results,
                            uint8_t* d_cigars, cudaStream_t st, int32_t max_len_sum) {
  AlignParams P;
  fill_params(h, b, P);
  P.results = d_results;
  P.cigars = d_cigars;
  if (P.compute_alignment && (!d_cigars || !b->cigar_off))
    return fail(h, WFA_ERR_ARGUMENT, "CIGAR output buffers are required in alignment scope");
  const int cls = metric_class(P.metric);
  const int nc = metric_components(P.metric);
  const bool packed = P.format == WFA_SEQ_PACKED2;
  const size_t smem = (size_t)kWarpsPerBlock * ring_desc_bytes(P.scope, nc);
  if (smem > 200 * 1024) return fail(h, WFA_ERR_UNSUPPORTED, "wavefront ring too large");
  const int occ = occupancy_blocks_per_sm(cls, packed, smem);

  ScratchCfg cfg;
  cfg.wmax = std::max(8, std::min(max_len_sum + 3, 8192));
  cfg.hist_scores = P.compute_alignment ? 1024 : 0;
  cfg.hist_words = P.compute_alignment ? (int64_t)std::max(32768, 16 * (max_len_sum + 3)) : 0;

  CUDA_TRY(h, h->counters.ensure(64), "counters");
  unsigned long long* d_work = h->counters.as<unsigned long long>();
  int32_t* d_retry = reinterpret_cast<int32_t*>(d_work + 1);

  int64_t todo = b->num_pairs;
  const int64_t* list = nullptr;
  h->last_kernel_ms = 0.0;
  const size_t budget = (size_t)6 << 30;  // scratch bytes per handle
  for (int round = 0; todo > 0; ++round) {
    if (round > 8) return fail(h, WFA_ERR_OOM, "alignment needs more scratch than available");
    int64_t ring_words = ((int64_t)P.scope * nc * cfg.wmax + 3) & ~(int64_t)3;
    int64_t warp_words = ring_words + (int64_t)cfg.hist_scores * 4 + cfg.hist_words;
    warp_words = (warp_words + 63) & ~(int64_t)63;
    int64_t max_warps = (int64_t)h->num_sms * occ * kWarpsPerBlock;
    int64_t warps = std::min<int64_t>(max_warps, (todo + 0) * 1);
    warps = std::max<int64_t>(warps, 1);
    while (warps > kWarpsPerBlock && (size_t)warps * warp_words * 4 > budget) warps /= 2;
    int blocks = (int)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
    size_t scratch_bytes = (size_t)blocks * kWarpsPerBlock * warp_words * 4;
    CUDA_TRY(h, h->scratch.ensure(scratch_bytes), "scratch");
    P.scratch = h->scratch.as<int32_t>();
    P.warp_words = warp_words;
    P.wmax = cfg.wmax;
    P.hist_scores = cfg.hist_scores;
    P.hist_words = cfg.hist_words;
    P.work_counter = d_work;
    P.retry_count = d_retry;
    P.pair_list = list;
    P.num_pairs = todo;
    CUDA_TRY(h, cudaMemsetAsync(d_work, 0, 16, st), "memset");
    CUDA_TRY(h, cudaEventRecord(h->ev0, st), "event");
    CUDA_TRY(h, launch_unialign(P, cls, blocks, smem, st), "kernel launch");
    CUDA_TRY(h, cudaEventRecord(h->ev1, st), "event");
    h->launches++;
    int32_t retries = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&retries, d_retry, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "kernel");
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
    h->last_kernel_ms += ms;
    if (retries == 0) break;
    // Gather the pairs to re-run into a list (double-buffered in pairlist).
    size_t lbytes = (size_t)retries * 8;
    CUDA_TRY(h, h->pairlist.ensure(2 * std::max(lbytes, (size_t)b->num_pairs * 8)), "pair list");
    int64_t* half0 = h->pairlist.as<int64_t>();
    int64_t* half1 = half0 + b->num_pairs;
    int64_t* out = (list == half0) ? half1 : half0;
    CUDA_TRY(h, cudaMemsetAsync(d_retry, 0, 4, st), "memset");
    int tb = 256;
    collect_retries<<<(unsigned)((todo + tb - 1) / tb), tb, 0, st>>>(d_results, list, todo, out, d_retry);
    h->launches++;
    CUDA_TRY(h, cudaGetLastError(), "collect retries");
    int32_t got = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&got, d_retry, 4, cudaMemcpyDeviceToHost, st), "retry count");
    CUDA_TRY(h, cudaStreamSynchronize(st), "collect retries");
    list = out;
    todo = got;
    cfg.wmax = std::min(max_len_sum + 3, std::max(cfg.wmax, 1) * 4);
    if (P.compute_alignment) {
      cfg.hist_scores *= 4;
      cfg.hist_words *= 4;
    }
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
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    delete h;
    if (err) *err = WFA_ERR_CUDA;
    return nullptr;
  }
  if (err) *err = WFA_OK;
  return h;
}

void wfa_aligner_destroy(wfa_aligner_t* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (DevBuf* b : {&h->seq, &h->poff, &h->plen, &h->toff, &h->tlen, &h->coff, &h->results,
                    &h->cigars, &h->dense, &h->scratch, &h->counters, &h->pairlist})
    b->release();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
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

// One pair through the batch path (plain per-call form).
static int32_t align_plain(wfa_aligner_t* h, const uint8_t* p, int32_t n, const uint8_t* t,
                           int32_t m, int span, bool packed) {
  if (!h || n < 0 || m < 0 || (n > 0 && !p) || (m > 0 && !t)) return WFA_ERR_ARGUMENT;
  h->last_err = WFA_OK;
  h->status = WFA_STATUS_OOM;
  h->cigar.clear();
  int saved_span = h->span;
  h->span = span;
  int r = check_supported(h, false);
  h->span = saved_span;
  if (r != WFA_OK) return r;
  cudaSetDevice(h->device);
  cudaStream_t st = h->stream;
  // Layout: pattern then text, each starting on a 16-byte boundary.
  size_t pbytes = packed ? ((size_t)n + 3) / 4 : (size_t)n;
  size_t tbytes = packed ? ((size_t)m + 3) / 4 : (size_t)m;
  size_t toff_b = (pbytes + 15) & ~(size_t)15;
  size_t total = toff_b + ((tbytes + 15) & ~(size_t)15) + 16;
  int64_t cap = 2 * ((int64_t)n + m) + 1;
  struct Meta { int64_t poff, toff, coff; int32_t plen, tlen; } meta;
  meta.poff = 0;
  meta.toff = packed ? (int64_t)(toff_b / 4) : (int64_t)toff_b;
  meta.coff = 0;
  meta.plen = n;
  meta.tlen = m;
  CUDA_TRY(h, h->seq.ensure(total), "seq");
  CUDA_TRY(h, h->poff.ensure(64), "meta");
  CUDA_TRY(h, h->results.ensure(sizeof(wfa_result_t)), "results");
  CUDA_TRY(h, h->cigars.ensure((size_t)cap), "cigars");
  std::vector<uint8_t> staging(total, 0);
  if (pbytes) std::memcpy(staging.data(), p, pbytes);
  if (tbytes) std::memcpy(staging.data() + toff_b, t, tbytes);
  CUDA_TRY(h, cudaMemcpyAsync(h->seq.p, staging.data(), total, cudaMemcpyHostToDevice, st), "H2D");
  CUDA_TRY(h, cudaMemcpyAsync(h->poff.p, &meta, sizeof meta, cudaMemcpyHostToDevice, st), "H2D");
  const char* mb = h->poff.as<char>();
  wfa_batch_t b;
  b.format = packed ? WFA_SEQ_PACKED2 : WFA_SEQ_ASCII;
  b.span = span;
  b.num_pairs = 1;
  b.seq = h->seq.p;
  b.seq_bytes = (int64_t)total;
  b.p_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, poff));
  b.t_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, toff));
  b.cigar_off = reinterpret_cast<const int64_t*>(mb + offsetof(Meta, coff));
  b.p_len = reinterpret_cast<const int32_t*>(mb + offsetof(Meta, plen));
  b.t_len = reinterpret_cast<const int32_t*>(mb + offsetof(Meta, tlen));
  b.cigar_bytes = cap;
  r = run_device_batch(h, &b, h->results.as<wfa_result_t>(), h->cigars.as<uint8_t>(), st, n + m);
  if (r != WFA_OK) return r;
  wfa_result_t res;
  CUDA_TRY(h, cudaMemcpyAsync(&res, h->results.p, sizeof res, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  if (res.cigar_length > 0) {
    h->cigar.resize((size_t)res.cigar_length);
    CUDA_TRY(h, cudaMemcpy(h->cigar.data(), h->cigars.as<uint8_t>() + res.cigar_begin,
                           (size_t)res.cigar_length, cudaMemcpyDeviceToHost), "D2H");
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
int32_t wfa_align_biwfa(wfa_aligner_t* h, const uint8_t*, int32_t, const uint8_t*, int32_t) {
  if (!h) return WFA_ERR_ARGUMENT;
  return check_supported(h, true);
}
int32_t wfa_align_biwfa_score(wfa_aligner_t* h, const uint8_t*, int32_t, const uint8_t*, int32_t) {
  if (!h) return WFA_ERR_ARGUMENT;
  return check_supported(h, true);
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
double wfa_last_kernel_ms(const wfa_aligner_t* h) { return h ? h->last_kernel_ms : 0.0; }

static int batch_common(wfa_aligner_t* h, const wfa_batch_t* b) {
  if (!h || !b || b->num_pairs < 0 || !b->seq || !b->p_off || !b->p_len || !b->t_off || !b->t_len)
    return WFA_ERR_ARGUMENT;
  if (b->format != WFA_SEQ_ASCII && b->format != WFA_SEQ_PACKED2) return WFA_ERR_ARGUMENT;
  if (b->span != WFA_SPAN_END2END && b->span != WFA_SPAN_ENDSFREE) return WFA_ERR_ARGUMENT;
  h->last_err = WFA_OK;
  int saved = h->span;
  h->span = b->span;
  int r = check_supported(h, false);
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
  CUDA_TRY(h, cudaMemsetAsync(d_max, 0, 4, st), "memset");
  max_lengths<<<256, 256, 0, st>>>(b->p_len, b->t_len, b->num_pairs, d_max);
  h->launches++;
  CUDA_TRY(h, cudaGetLastError(), "max lengths");
  int32_t mx = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&mx, d_max, 4, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "max lengths");
  return run_device_batch(h, b, results, cigars, st, mx);
}

int wfa_batch_align(wfa_aligner_t* h, const wfa_batch_t* b, wfa_result_t* results, uint8_t* cigars) {
  int r = batch_common(h, b);
  if (r != WFA_OK) return r;
  if (!results) return WFA_ERR_ARGUMENT;
  const int64_t n = b->num_pairs;
  if (n == 0) return WFA_OK;
  const bool aln = h->scope == WFA_SCOPE_ALIGNMENT;
  if (aln && !cigars) return WFA_ERR_ARGUMENT;
  cudaSetDevice(h->device);
  cudaStream_t st = h->stream;
  int32_t mx = 0;
  int64_t slot_total = 0;
  std::vector<int64_t> slot_off;
  if (aln) slot_off.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    int32_t s = b->p_len[i] + b->t_len[i];
    mx = std::max(mx, s);
    if (aln) {
      slot_off[(size_t)i] = slot_total;
      slot_total += 2 * (int64_t)s + 1;
    }
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
  d.p_off = h->poff.as<int64_t>();
  d.t_off = h->toff.as<int64_t>();
  d.p_len = h->plen.as<int32_t>();
  d.t_len = h->tlen.as<int32_t>();
  d.cigar_off = nullptr;
  if (aln) {
    CUDA_TRY(h, h->coff.ensure((size_t)n * 8), "cigar_off");
    CUDA_TRY(h, h->cigars.ensure((size_t)slot_total + 16), "cigar slots");
    CUDA_TRY(h, cudaMemcpyAsync(h->coff.p, slot_off.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
    d.cigar_off = h->coff.as<int64_t>();
    d.cigar_bytes = slot_total;
  }
  r = run_device_batch(h, &d, h->results.as<wfa_result_t>(), aln ? h->cigars.as<uint8_t>() : nullptr, st, mx);
  if (r != WFA_OK) return r;
  CUDA_TRY(h, cudaMemcpyAsync(results, h->results.p, (size_t)n * sizeof(wfa_result_t),
                              cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  if (!aln) return WFA_OK;
  // Dense CIGAR packing in input order: results[i].cigar_begin becomes the
  // offset of pair i's ops in `cigars`.
  std::vector<int64_t> dst((size_t)n);
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) {
    dst[(size_t)i] = total;
    total += results[i].cigar_length;
  }
  CUDA_TRY(h, h->dense.ensure((size_t)total + 16), "dense cigars");
  CUDA_TRY(h, h->pairlist.ensure((size_t)n * 8), "offsets");
  CUDA_TRY(h, cudaMemcpyAsync(h->pairlist.p, dst.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st), "H2D");
  int64_t threads = n * 32;
  compact_cigars<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      h->results.as<wfa_result_t>(), d.cigar_off, h->cigars.as<uint8_t>(), h->pairlist.as<int64_t>(),
      h->dense.as<uint8_t>(), n);
  h->launches++;
  CUDA_TRY(h, cudaGetLastError(), "compact cigars");
  CUDA_TRY(h, cudaMemcpyAsync(cigars, h->dense.p, (size_t)total, cudaMemcpyDeviceToHost, st), "D2H");
  CUDA_TRY(h, cudaStreamSynchronize(st), "D2H");
  for (int64_t i = 0; i < n; ++i) results[i].cigar_begin = (int32_t)dst[(size_t)i];
  return WFA_OK;
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
