// wfa_oracle.cpp -- CPU oracle: a C++ restatement of the wfa2lib-rs alignment
// path.  TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline); the
// product library never links it.
//
// Every function cites the reference item it restates (paths are relative to
// the wfa2lib-rs project root).  The restatement keeps the reference's
// wavefront semantics literally -- per-wavefront allocation ranges,
// initialised ranges, NULL padding of input ends, null/victim wavefronts --
// so that its results (scores, CIGARs, tie-breaks, statuses) are the
// reference's, and so that the CUDA path's simpler storage model is checked
// against the literal one.  With -DWFO_CHECKS every read of a cell that the
// reference never initialised aborts (poisoned memory).
//
// Not restated here (out of the hot path or later rows): lambda sequences
// (host callback), Compat::Corrected.

#include "wfa_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#ifdef WFO_CHECKS
#define WFO_ASSERT(c)                                                              \
  do {                                                                             \
    if (!(c)) {                                                                    \
      std::fprintf(stderr, "oracle check failed %s:%d: %s\n", __FILE__, __LINE__, #c); \
      std::abort();                                                                \
    }                                                                              \
  } while (0)
#else
#define WFO_ASSERT(c) ((void)0)
#endif

namespace wfo {

// src/offset.rs:15, src/offset.rs:46
constexpr int32_t OFFSET_NULL = INT32_MIN / 2;
constexpr int32_t DIAG_NULL = INT32_MAX;
// Marker for cells the reference leaves uninitialised.
constexpr int32_t POISON = INT32_MIN + 0x5A5A;

enum Metric { INDEL = 0, EDIT = 1, LINEAR = 2, AFFINE = 3, AFFINE2P = 4 };
enum Status { OK = 0, END_REACHED, END_UNREACHABLE, MAX_STEPS, OOM, COMPLETED, PARTIAL };
enum Comp { CM = 0, CI1 = 1, CD1 = 2, CI2 = 3, CD2 = 4 };
enum Heur { H_NONE = 0, H_WFADAPTIVE, H_XDROP, H_ZDROP, H_BANDED_STATIC, H_BANDED_ADAPTIVE };

static inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wrap_sub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static inline int32_t wrap_mul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

// ---------------------------------------------------------------------------
// Penalties: src/penalties.rs:119-296
// ---------------------------------------------------------------------------
struct Penalties {
  int metric = AFFINE;
  int32_t match_ = 0, mismatch = 0, o1 = 0, e1 = 0, o2 = -1, e2 = -1;
  int32_t orig[6] = {0, 0, 0, 0, 0, 0};  // user penalties (match first)
  int32_t internal_gap_e = 0;

  // WavefrontPenalties::wf_score_to_sw_score, src/penalties.rs:300-308
  int32_t wf_score_to_sw_score(int32_t plen, int32_t tlen, int32_t s) const {
    int32_t swg_match = -match_;
    return wrap_sub(wrap_mul(swg_match, wrap_add(plen, tlen)), s) / 2;
  }
};

static bool make_penalties(int metric, const int32_t* p, Penalties& out) {
  Penalties r;
  r.metric = metric;
  switch (metric) {
    case INDEL:  // new_indel :119
      r.match_ = 0; r.mismatch = -1; r.o1 = 1; r.e1 = -1; r.internal_gap_e = 1;
      break;
    case EDIT:  // new_edit :137
      r.match_ = 0; r.mismatch = 1; r.o1 = 1; r.e1 = -1; r.internal_gap_e = 1;
      break;
    case LINEAR: {  // new_linear :157-186
      int32_t m = p[0], x = p[1], i = p[2];
      if (m > 0 || !(x > 0 && i > 0)) return false;
      if (m < 0) { r.match_ = m; r.mismatch = 2 * x - 2 * m; r.o1 = 2 * i - m; }
      else { r.match_ = 0; r.mismatch = x; r.o1 = i; }
      r.e1 = -1; r.internal_gap_e = i;
      for (int q = 0; q < 3; ++q) r.orig[q] = p[q];
      break;
    }
    case AFFINE: {  // new_affine :192-235
      int32_t m = p[0], x = p[1], o = p[2], e = p[3];
      if (m > 0 || !(x > 0 && o >= 0 && e > 0)) return false;
      if (m < 0) { r.match_ = m; r.mismatch = 2 * x - 2 * m; r.o1 = 2 * o; r.e1 = 2 * e - m; }
      else { r.match_ = 0; r.mismatch = x; r.o1 = o; r.e1 = e; }
      r.internal_gap_e = e;
      for (int q = 0; q < 4; ++q) r.orig[q] = p[q];
      break;
    }
    case AFFINE2P: {  // new_affine2p :241-296
      int32_t m = p[0], x = p[1], o1 = p[2], e1 = p[3], o2 = p[4], e2 = p[5];
      if (m > 0 || !(x > 0 && o1 >= 0 && e1 > 0 && o2 >= 0 && e2 > 0)) return false;
      if (m < 0) {
        r.match_ = m; r.mismatch = 2 * x - 2 * m; r.o1 = 2 * o1; r.e1 = 2 * e1 - m;
        r.o2 = 2 * o2; r.e2 = 2 * e2 - m;
      } else {
        r.match_ = 0; r.mismatch = x; r.o1 = o1; r.e1 = e1; r.o2 = o2; r.e2 = e2;
      }
      r.internal_gap_e = e1;
      for (int q = 0; q < 6; ++q) r.orig[q] = p[q];
      break;
    }
    default:
      return false;
  }
  out = r;
  return true;
}

// ---------------------------------------------------------------------------
// CIGAR: src/cigar.rs
// ---------------------------------------------------------------------------
struct Cigar {
  std::vector<uint8_t> ops;
  int64_t begin = 0, end = 0;
  int32_t score = INT32_MIN, end_v = -1, end_h = -1;

  void clear() { begin = 0; end = 0; score = INT32_MIN; end_v = -1; end_h = -1; }  // :45
  void resize(size_t n) {  // :54
    if (n > ops.size()) ops.assign(n, 0);
    clear();
  }
  bool empty() const { return begin >= end; }
  void append_forward(const Cigar& o) {  // :79
    for (int64_t i = o.begin; i < o.end; ++i) ops[end++] = o.ops[i];
  }
  void append_deletion(int64_t n) { for (int64_t i = 0; i < n; ++i) ops[end++] = 'D'; }
  void append_insertion(int64_t n) { for (int64_t i = 0; i < n; ++i) ops[end++] = 'I'; }

  int32_t score_edit() const {  // :113
    int32_t s = 0;
    for (int64_t i = begin; i < end; ++i) s += ops[i] != 'M';
    return s;
  }
  int32_t score_gap_linear(const int32_t* p) const {  // :126 (p = match, x, indel)
    int32_t s = 0;
    for (int64_t i = begin; i < end; ++i) {
      uint8_t op = ops[i];
      if (op == 'M') s -= p[0];
      else if (op == 'X') s -= p[1];
      else s -= p[2];
    }
    return s;
  }
  int32_t score_gap_affine(const int32_t* p) const {  // :139 (match, x, o, e)
    int32_t s = 0;
    uint8_t last = 0;
    for (int64_t i = begin; i < end; ++i) {
      uint8_t op = ops[i];
      if (op == 'M') s -= p[0];
      else if (op == 'X') s -= p[1];
      else if (op == 'D') s -= p[3] + (last == 'D' ? 0 : p[2]);
      else s -= p[3] + (last == 'I' ? 0 : p[2]);
      last = op;
    }
    return s;
  }
  static int32_t affine2p_op(uint8_t op, int32_t len, const int32_t* p) {  // :189
    if (op == 'M') return p[0] * len;
    if (op == 'X') return p[1] * len;
    int32_t s1 = p[2] + p[3] * len, s2 = p[4] + p[5] * len;
    return std::min(s1, s2);
  }
  int32_t score_gap_affine2p(const int32_t* p) const {  // :171
    int32_t s = 0, len = 0;
    uint8_t last = 0;
    for (int64_t i = begin; i < end; ++i) {
      uint8_t op = ops[i];
      if (op != last && last != 0) { s -= affine2p_op(last, len, p); len = 0; }
      last = op;
      ++len;
    }
    if (last != 0) s -= affine2p_op(last, len, p);
    return s;
  }

  // maxtrim_gap_linear / maxtrim_gap_affine, src/cigar.rs:207-334.
  bool maxtrim_simple(const int32_t* p, bool affine) {
    int64_t b = begin, e = end;
    if (b >= e) return false;
    int32_t match_score = p[0] != 0 ? p[0] : -1;
    int32_t max_score = 0, max_v = 0, max_h = 0;
    int64_t max_off = b;
    int32_t s = 0, v = 0, h = 0;
    uint8_t last = 0;
    for (int64_t i = b; i < e; ++i) {
      uint8_t op = ops[i];
      switch (op) {
        case 'M': s -= match_score; ++v; ++h; break;
        case 'X': s -= p[1]; ++v; ++h; break;
        case 'I':
          s -= affine ? p[3] + (last == 'I' ? 0 : p[2]) : p[2];
          ++h;
          break;
        case 'D':
          s -= affine ? p[3] + (last == 'D' ? 0 : p[2]) : p[2];
          ++v;
          break;
        default: break;
      }
      last = op;
      if (max_score < s) { max_score = s; max_off = i; max_v = v; max_h = h; }
    }
    bool trimmed = max_off != e - 1;
    if (max_score == 0) clear();
    else { end = max_off + 1; score = max_score; end_v = max_v; end_h = max_h; }
    return trimmed;
  }
  static int32_t maxtrim_2p_op(uint8_t op, int32_t len, const int32_t* p, int32_t& v, int32_t& h) {
    switch (op) {  // :424
      case 'M': v += len; h += len; return (p[0] != 0 ? p[0] : -1) * len;
      case 'X': v += len; h += len; return p[1] * len;
      case 'D': v += len; return std::min(p[2] + p[3] * len, p[4] + p[5] * len);
      case 'I': h += len; return std::min(p[2] + p[3] * len, p[4] + p[5] * len);
      default: return 0;
    }
  }
  bool maxtrim_gap_affine2p(const int32_t* p) {  // :349
    int64_t b = begin, e = end;
    if (b >= e) return false;
    int32_t max_score = 0, max_v = 0, max_h = 0;
    int64_t max_off = b;
    uint8_t last = 0;
    int32_t s = 0, v = 0, h = 0, len = 0;
    for (int64_t i = b; i < e; ++i) {
      uint8_t op = ops[i];
      if (op != last && last != 0) {
        s -= maxtrim_2p_op(last, len, p, v, h);
        len = 0;
        if (max_score < s) { max_score = s; max_off = i - 1; max_v = v; max_h = h; }
      }
      last = op;
      ++len;
    }
    s -= maxtrim_2p_op(last, len, p, v, h);
    if (max_score < s) { max_score = s; max_off = e - 1; max_v = v; max_h = h; }
    bool trimmed = max_off != e - 1;
    if (max_score == 0) clear();
    else { end = max_off + 1; score = max_score; end_v = max_v; end_h = max_h; }
    return trimmed;
  }

  // to_string_rle(true), src/cigar.rs:522-546
  std::string rle() const {
    std::string r;
    if (empty()) return r;
    uint8_t last = ops[begin];
    int64_t n = 1;
    char tmp[32];
    for (int64_t i = begin + 1; i < end; ++i) {
      if (ops[i] == last) { ++n; continue; }
      std::snprintf(tmp, sizeof tmp, "%lld%c", (long long)n, last);
      r += tmp;
      last = ops[i];
      n = 1;
    }
    std::snprintf(tmp, sizeof tmp, "%lld%c", (long long)n, last);
    r += tmp;
    return r;
  }
};

// ---------------------------------------------------------------------------
// Sequences: src/sequences.rs:153-205 (ASCII, padded, sentinels '!' / '?')
// ---------------------------------------------------------------------------
struct Sequences {
  static constexpr size_t PAD = 64;
  std::vector<uint8_t> buf;
  size_t pstart = 0, tstart = 0;
  int32_t plen = 0, tlen = 0;

  void init_ascii(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m, bool reverse) {
    size_t need = (size_t)n + (size_t)m + 3 * PAD;
    if (buf.size() < need) buf.assign(need + need / 2, 0);
    pstart = PAD;
    tstart = PAD + (size_t)n + PAD;
    for (int32_t i = 0; i < n; ++i) buf[pstart + i] = reverse ? p[n - 1 - i] : p[i];
    buf[pstart + n] = '!';
    for (int32_t i = 0; i < m; ++i) buf[tstart + i] = reverse ? t[m - 1 - i] : t[i];
    buf[tstart + m] = '?';
    plen = n;
    tlen = m;
  }
  const uint8_t* P() const { return buf.data() + pstart; }
  const uint8_t* T() const { return buf.data() + tstart; }
  bool cmp(int32_t v, int32_t h) const { return P()[v] == T()[h]; }
};

// decode_packed2bits, src/sequences.rs:34-52
static std::vector<uint8_t> decode_packed2bits(const uint8_t* packed, int32_t len) {
  static const char dna[4] = {'A', 'C', 'G', 'T'};
  std::vector<uint8_t> r((size_t)len);
  for (int32_t i = 0; i < len; ++i) r[i] = dna[(packed[i >> 2] >> (2 * (i & 3))) & 3];
  return r;
}

// ---------------------------------------------------------------------------
// Wavefront: src/wavefront.rs (allocation range, limits, initialised range)
// ---------------------------------------------------------------------------
struct Wavefront {
  std::vector<int32_t> mem;
  int32_t base_k = 0, alloc = 0;
  int32_t lo = 1, hi = -1, init_min = 0, init_max = 0;
  bool null = false;
  // Med/low (piggyback) bookkeeping, src/wavefront.rs:359-415: the range of
  // cells whose backtrace was written since init (a union range, as the
  // reference keeps it) and the begin-free seeds placed in this wavefront.
  int32_t wr_lo = 1, wr_hi = 0;
  std::vector<int32_t> seeds;
  // The piggyback kernels' per-cell backtrace (src/wavefront.rs:64-77,
  // 529-580): the packed CIGAR (up to 16 operations, src/pcigar.rs) and the
  // index of the backtrace-buffer block it continues; and the occupancy the
  // offload tracks (bt_occupancy_max).  Sized with the offsets when an
  // aligner runs the literal piggyback path, else empty.
  std::vector<uint32_t> pc, pvb;
  int32_t occ = 0;
  bool has_bt() const { return !pc.empty(); }
  void ensure_bt() {  // fresh arrays are zeroed (alloc_zeroed, :283-301)
    if (pc.size() != mem.size()) { pc.assign(mem.size(), 0); pvb.assign(mem.size(), 0); }
  }
  uint32_t get_pc(int32_t k) const { WFO_ASSERT(allocated(k)); return pc[(size_t)(k - base_k)]; }
  uint32_t get_pv(int32_t k) const { WFO_ASSERT(allocated(k)); return pvb[(size_t)(k - base_k)]; }
  void set_bt(int32_t k, uint32_t c, uint32_t v) {
    WFO_ASSERT(allocated(k));
    pc[(size_t)(k - base_k)] = c;
    pvb[(size_t)(k - base_k)] = v;
  }
  // zero_bt, :570-580: zeroed backtraces count as written.
  void zero_bt(int32_t k, int32_t count) {
    if (!has_bt() || count <= 0) return;
    mark_written(k, k + count - 1);
    for (int32_t i = 0; i < count; ++i) set_bt(k + i, 0, 0);
  }
  // bt_or_zero, :410-416
  void bt_or_zero(int32_t k, uint32_t& c, uint32_t& v) const {
    if (!written(k)) { c = 0; v = 0; return; }
    c = get_pc(k);
    v = get_pv(k);
  }
  void mark_written(int32_t l, int32_t h) {
    if (l > h) return;
    if (wr_lo > wr_hi) { wr_lo = l; wr_hi = h; }
    else { wr_lo = std::min(wr_lo, l); wr_hi = std::max(wr_hi, h); }
  }
  bool written(int32_t k) const { return k >= wr_lo && k <= wr_hi; }
  bool is_seed(int32_t k) const { return std::find(seeds.begin(), seeds.end(), k) != seeds.end(); }

  bool allocated(int32_t k) const { return k >= base_k && k < base_k + alloc; }
  int32_t get(int32_t k) const {
    WFO_ASSERT(allocated(k));
    int32_t v = mem[(size_t)(k - base_k)];
    WFO_ASSERT(v != POISON);
    return v;
  }
  void set(int32_t k, int32_t v) {
    WFO_ASSERT(allocated(k));
    mem[(size_t)(k - base_k)] = v;
  }
  void fill_null(int32_t from, int32_t count) {
    for (int32_t i = 0; i < count; ++i) set(from + i, OFFSET_NULL);
  }
  void reallocate(int32_t n) {  // Wavefront::resize :283 (content lost)
    alloc = n;
#ifdef WFO_CHECKS
    mem.assign((size_t)n, POISON);  // never-initialised cells are detectable
#else
    mem.resize((size_t)n);
#endif
    if (has_bt()) { pc.assign((size_t)n, 0); pvb.assign((size_t)n, 0); }
  }
  void init(int32_t min_lo, int32_t /*max_hi*/) {  // :307
    null = false; lo = 1; hi = -1; base_k = min_lo; init_min = 0; init_max = 0;
    wr_lo = 1; wr_hi = 0; seeds.clear(); occ = 0;
  }
  void init_null(int32_t min_lo, int32_t max_hi) {  // :331
    null = true; lo = 1; hi = -1; base_k = min_lo; wr_lo = 1; wr_hi = 0; seeds.clear(); occ = 0;
    for (int32_t i = 0; i < max_hi - min_lo + 1; ++i) mem[(size_t)i] = OFFSET_NULL;
    if (has_bt())
      for (int32_t i = 0; i < max_hi - min_lo + 1; ++i) { pc[(size_t)i] = 0; pvb[(size_t)i] = 0; }
    init_min = min_lo; init_max = max_hi;
  }
  void init_victim(int32_t min_lo, int32_t max_hi) { init(min_lo, max_hi); null = true; }
  void set_limits(int32_t l, int32_t h) {  // :360
    lo = l; hi = h; init_min = l; init_max = h;
    mark_written(l, h);
  }
  void clear_init_range() { init_min = lo; init_max = hi; }  // :375
  void set_null_cell_if_allocated(int32_t k) {  // :395-405
    if (allocated(k)) { set(k, OFFSET_NULL); zero_bt(k, 1); }
  }
  void init_ends_lower(int32_t min_lo) {  // :422
    if (init_min <= min_lo) return;
    int32_t min_init = std::min(init_min, lo);
    int32_t start = std::max(min_lo, base_k);
    if (start < min_init) { fill_null(start, min_init - start); zero_bt(start, min_init - start); }
    init_min = start;
  }
  void init_ends_higher(int32_t max_hi) {  // :443
    if (init_max >= max_hi) return;
    int32_t max_init = std::max(init_max, hi);
    int32_t end = std::min(max_hi, base_k + alloc - 1);
    if (end > max_init) { fill_null(max_init + 1, end - max_init); zero_bt(max_init + 1, end - max_init); }
    init_max = end;
  }
};

// trim_ends, src/compute/mod.rs:14-49
static void trim_ends(int32_t plen, int32_t tlen, Wavefront& wf) {
  int32_t lo = wf.lo, k = wf.hi;
  while (k >= lo) {
    int32_t off = wf.get(k);
    if ((uint32_t)off <= (uint32_t)tlen && (uint32_t)(off - k) <= (uint32_t)plen) break;
    --k;
  }
  wf.hi = k;
  wf.init_max = k;
  int32_t hi = wf.hi;
  k = wf.lo;
  while (k <= hi) {
    int32_t off = wf.get(k);
    if ((uint32_t)off <= (uint32_t)tlen && (uint32_t)(off - k) <= (uint32_t)plen) break;
    ++k;
  }
  wf.lo = k;
  wf.init_min = k;
  wf.null = wf.lo > wf.hi;
}

// ---------------------------------------------------------------------------
// Heuristics: src/heuristic.rs
// ---------------------------------------------------------------------------
struct Heuristic {
  int kind = H_NONE;
  int32_t p0 = 0, p1 = 0, p2 = 0;
  // WfAdaptive (min_wf_len, max_distance, steps); XDrop/ZDrop (drop, steps);
  // BandedStatic (min_k, max_k); BandedAdaptive (min_k, max_k, steps).
  int32_t steps() const {
    switch (kind) {
      case H_WFADAPTIVE: case H_BANDED_ADAPTIVE: return p2;
      case H_XDROP: case H_ZDROP: return p1;
      default: return 0;
    }
  }
  bool banded() const { return kind == H_BANDED_STATIC || kind == H_BANDED_ADAPTIVE; }
  Heuristic with_band(int32_t min_k, int32_t max_k) const {  // src/aligner.rs:330-343
    Heuristic h = *this;
    if (banded()) { h.p0 = min_k; h.p1 = max_k; }
    return h;
  }
};

struct HeurState {  // src/heuristic.rs:62-148
  int32_t steps_wait = 0, max_sw_score = 0, max_wf_score = 0;
  int32_t max_sw_score_k = DIAG_NULL, max_sw_score_offset = OFFSET_NULL, zdrop_last_score = 0;
  void reset(const Heuristic& h) { *this = HeurState(); steps_wait = h.steps(); }
};

struct DropParams {  // src/heuristic.rs:75-107
  int32_t swg_match = 1, pattern_begin_free = 0, text_begin_free = 0, max_penalty = 0;
};

// wf_distance_end2end, src/heuristic.rs:152-162
static inline int32_t wf_distance_end2end(int32_t off, int32_t k, int32_t plen, int32_t tlen) {
  if (off < 0) return INT32_MAX;
  return std::max(plen - (off - k), tlen - off);
}

// wfadaptive_reduce, src/heuristic.rs:312-345
static void wfadaptive_reduce(Wavefront& wf, const std::vector<int32_t>& d, int32_t dbase,
                              int32_t min_distance, int32_t thr, int32_t min_k, int32_t max_k) {
  int32_t top_limit = std::min(max_k, wf.hi);
  int32_t lo_reduced = wf.lo;
  for (int32_t k = wf.lo; k < top_limit; ++k) {
    if (wrap_sub(d[(size_t)(k - dbase)], min_distance) <= thr) break;
    ++lo_reduced;
  }
  wf.lo = lo_reduced;
  int32_t bottom_limit = std::max(min_k, wf.lo);
  int32_t hi_reduced = wf.hi;
  for (int32_t k = wf.hi; k > bottom_limit; --k) {
    if (wrap_sub(d[(size_t)(k - dbase)], min_distance) <= thr) break;
    --hi_reduced;
  }
  wf.hi = hi_reduced;
}

// compute_sw_scores, src/heuristic.rs:491-520
static void compute_sw_scores(const Wavefront& wf, std::vector<int32_t>& sw, int32_t base,
                              const DropParams& drop, int32_t wf_score, int32_t& cmax,
                              int32_t& cmax_k, int32_t& cmax_off) {
  cmax = INT32_MIN; cmax_k = 0; cmax_off = 0;
  for (int32_t k = wf.lo; k <= wf.hi; ++k) {
    int32_t off = wf.get(k);
    if (off < 0) continue;
    int32_t free_v = k < 0 ? std::min(-k, drop.pattern_begin_free) : 0;
    int32_t free_h = k > 0 ? std::min(k, drop.text_begin_free) : 0;
    int32_t v = off - k - free_v, h = off - free_h;
    int32_t s = (drop.swg_match * (v + h) - wf_score) / 2;
    sw[(size_t)(k - base)] = s;
    if (cmax < s) { cmax = s; cmax_k = k; cmax_off = off; }
  }
}

// heuristic_cutoff, src/heuristic.rs:167-254 (and the per-strategy cutoffs)
static bool heuristic_cutoff(const Heuristic& hs, HeurState& st, Wavefront& wf,
                             std::vector<int32_t>& scratch, int32_t sbase, int32_t plen,
                             int32_t tlen, const DropParams& drop, int32_t score) {
  if (wf.lo > wf.hi) return false;
  st.steps_wait -= 1;
  switch (hs.kind) {
    case H_WFADAPTIVE: {  // :258-309
      if (st.steps_wait > 0) return false;
      int32_t blo = wf.lo, bhi = wf.hi;
      if (bhi - blo + 1 < hs.p0) return false;
      int32_t min_d = std::max(plen, tlen);
      for (int32_t k = blo; k <= bhi; ++k) {
        int32_t d = wf_distance_end2end(wf.get(k), k, plen, tlen);
        scratch[(size_t)(k - sbase)] = d;
        if (d < min_d) min_d = d;
      }
      int32_t ak = tlen - plen;
      wfadaptive_reduce(wf, scratch, sbase, min_d, hs.p1, ak, ak);
      st.steps_wait = hs.p2;
      return false;
    }
    case H_BANDED_STATIC:  // :396
      if (wf.lo < hs.p0) wf.lo = hs.p0;
      if (wf.hi > hs.p1) wf.hi = hs.p1;
      return false;
    case H_BANDED_ADAPTIVE: {  // :355-393
      if (st.steps_wait > 0) return false;
      int32_t lo = wf.lo, hi = wf.hi, len = hi - lo + 1;
      if (len < 4) return false;
      int32_t maxlen = hs.p1 - hs.p0 + 1;
      if (len > maxlen) {
        int32_t leeway = (len - maxlen) / 2, quarter = len / 4;
        auto dist = [&](int32_t k) { return wf_distance_end2end(wf.get(k), k, plen, tlen); };
        int32_t d0 = dist(lo), d1 = dist(lo + quarter), d2 = dist(lo + 2 * quarter), d3 = dist(hi);
        int32_t new_lo = lo;
        if (d0 > d3) new_lo += leeway;
        if (d1 > d2) new_lo += leeway;
        wf.lo = std::max(new_lo, lo);
        wf.hi = std::min(new_lo + maxlen - 1, hi);
      }
      st.steps_wait = hs.p2;
      return false;
    }
    case H_XDROP: {  // :410-451
      if (st.steps_wait > 0) return false;
      int32_t cmax, ck, co;
      compute_sw_scores(wf, scratch, sbase, drop, score, cmax, ck, co);
      if (st.max_sw_score_k != DIAG_NULL) {
        int32_t mx = st.max_sw_score;
        auto drops = [&](int32_t k) { return mx - scratch[(size_t)(k - sbase)] >= hs.p0; };
        int32_t k = wf.lo;
        while (k <= wf.hi && (wf.get(k) < 0 || drops(k))) ++k;
        wf.lo = k;
        k = wf.hi;
        while (k >= wf.lo && (wf.get(k) < 0 || drops(k))) --k;
        wf.hi = k;
        if (cmax > st.max_sw_score) { st.max_sw_score = cmax; st.max_sw_score_k = ck; }
      } else {
        st.max_sw_score = cmax;
        st.max_sw_score_k = ck;
      }
      st.steps_wait = hs.p1;
      return false;
    }
    case H_ZDROP: {  // :456-486
      if (st.steps_wait > 0) return false;
      int32_t cmax, ck, co;
      compute_sw_scores(wf, scratch, sbase, drop, score, cmax, ck, co);
      if (st.max_sw_score_k == DIAG_NULL || cmax > st.max_sw_score) {
        st.max_sw_score = cmax; st.max_wf_score = score; st.max_sw_score_k = ck;
        st.max_sw_score_offset = co; st.zdrop_last_score = score;
      } else if (st.max_sw_score - cmax <= hs.p0) {
        st.zdrop_last_score = score;
      } else if (score - st.zdrop_last_score >= drop.max_penalty) {
        return true;
      }
      st.steps_wait = hs.p1;
      return false;
    }
    default:
      return false;
  }
}

// ---------------------------------------------------------------------------
// Components: src/components.rs (flat or modular per-score arrays)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// The piggyback backtrace of med/low memory, as the reference runs it:
// packed CIGARs (src/pcigar.rs:13-199) and the backtrace buffer
// (src/bt_buffer.rs:34-327).  Block indices are plain vector positions (the
// reference's segments are storage detail), and the buffer is never
// compacted here: compaction (:238-327) renumbers blocks without changing
// any chain's content, so results do not depend on it.
// ---------------------------------------------------------------------------
constexpr uint32_t PCIGAR_DELETION = 1, PCIGAR_MISMATCH = 2, PCIGAR_INSERTION = 3;
constexpr uint32_t PCIGAR_FULL_MASK = 0x40000000u, PCIGAR_ALMOST_FULL_MASK = 0x10000000u,
                   PCIGAR_HALF_FULL_MASK = 0x00010000u;
constexpr int32_t PCIGAR_MAX_LENGTH = 16;
constexpr uint32_t BT_BLOCK_IDX_NULL = 0xFFFFFFFFu;
static inline uint32_t pcigar_push(uint32_t pc, uint32_t op) { return (pc << 2) | op; }
static inline int32_t pcigar_free_slots(uint32_t pc) {  // :77-84
  return pc ? __builtin_clz(pc) / 2 : PCIGAR_MAX_LENGTH;
}

struct BtBuffer {
  std::vector<std::pair<uint32_t, uint32_t>> blocks;  // {pcigar, prev}
  std::vector<std::pair<int32_t, int32_t>> init_pos;  // {v, h}
  std::vector<uint32_t> packed;                       // traceback: end first
  void clear() { blocks.clear(); init_pos.clear(); }
  uint32_t store_block(uint32_t pc, uint32_t prev) {  // :112-131
    blocks.emplace_back(pc, prev);
    return (uint32_t)blocks.size() - 1;
  }
  uint32_t init_block(int32_t v, int32_t h) {  // :134-139
    init_pos.emplace_back(v, h);
    return store_block((uint32_t)init_pos.size() - 1, BT_BLOCK_IDX_NULL);
  }
  // traceback_from, :196-212: the pcigars back to the initial block (end
  // first); returns the initial block's pcigar (an index of init_pos).
  uint32_t traceback_from(uint32_t pc, uint32_t prev) {
    packed.clear();
    while (prev != BT_BLOCK_IDX_NULL) {
      packed.push_back(pc);
      const auto& b = blocks[prev];
      pc = b.first;
      prev = b.second;
    }
    return pc;
  }
};

struct Components {
  bool modular = false;
  size_t num_wavefronts = 0, scope = 0;
  int32_t hist_lo = 0, hist_hi = 0, alloc_lo = 0, alloc_hi = 0;
  std::vector<Wavefront*> arr[5];
  Wavefront null_wf, victim_wf;

  // compute_dimensions, src/components.rs:435-505
  static void dims(const Penalties& p, int32_t plen, int32_t tlen, bool modular, size_t& scope,
                   size_t& num) {
    int32_t absd = std::abs(plen - tlen);
    switch (p.metric) {
      case INDEL: case EDIT:
        scope = 2;
        num = modular ? 2
                      : (p.metric == INDEL ? (size_t)(plen + tlen) + 1
                                           : (size_t)std::max(plen, tlen) + 1);
        break;
      case LINEAR:
        scope = (size_t)std::max(p.mismatch, p.o1) + 1;
        num = modular ? scope : (size_t)(std::min(plen, tlen) * p.mismatch + p.o1 * absd + 1);
        break;
      case AFFINE:
        scope = (size_t)std::max(p.o1 + p.e1, p.mismatch) + 1;
        num = modular ? scope
                      : (size_t)(std::min(plen, tlen) * p.mismatch + p.o1 + absd * p.e1 + 1);
        break;
      default: {
        int32_t si = std::max(p.o1 + p.e1, p.o2 + p.e2);
        scope = (size_t)std::max(si, p.mismatch) + 1;
        int32_t i1 = p.o1 + absd * p.e1, i2 = p.o2 + absd * p.e2;
        num = modular ? scope : (size_t)(std::min(plen, tlen) * p.mismatch + std::min(i1, i2) + 1);
      }
    }
  }
  void create(int32_t plen, int32_t tlen, const Penalties& p, bool mod) {  // :93-131
    modular = mod;
    dims(p, plen, tlen, mod, scope, num_wavefronts);
    for (auto& a : arr) a.assign(num_wavefronts, nullptr);
    null_wf.reallocate(2049);
    null_wf.init_null(-1024, 1024);
    victim_wf.reallocate(2049);
    victim_wf.init_victim(-1024, 1024);
    hist_lo = hist_hi = alloc_lo = alloc_hi = 0;
  }
  void clear() {
    for (auto& a : arr) std::fill(a.begin(), a.end(), nullptr);
    hist_lo = hist_hi = alloc_lo = alloc_hi = 0;
  }
  void resize(int32_t plen, int32_t tlen, const Penalties& p) {  // :170-192
    size_t sc, num;
    dims(p, plen, tlen, modular, sc, num);
    scope = sc;
    if (num > num_wavefronts) {
      num_wavefronts = num;
      for (auto& a : arr) a.assign(num_wavefronts, nullptr);
      hist_lo = hist_hi = alloc_lo = alloc_hi = 0;
    } else {
      clear();
    }
  }
  void resize_null_victim(int32_t lo, int32_t hi) {  // :195-211
    if (lo - 1 < null_wf.init_min || hi + 1 > null_wf.init_max) {
      int32_t len = hi - lo + 1, inc = (len * 3) / 2;
      int32_t plo = lo - inc / 2, phi = hi + inc / 2;
      victim_wf.reallocate(phi - plo + 1);
      victim_wf.init_victim(plo, phi);
      null_wf.reallocate(phi - plo + 1);
      null_wf.init_null(plo, phi);
    }
  }
  size_t slot(int32_t score) const {
    return modular ? (size_t)((uint32_t)score % (uint32_t)scope) : (size_t)score;
  }
  bool has_slot(int32_t score) const { return modular || (size_t)score < num_wavefronts; }
  // Med/low keep every score here (the reference's modular components have
  // no score cap): the arrays grow on demand.
  bool grow = false;
  bool make_slot(int32_t score) {
    if (grow && !modular && (size_t)score >= num_wavefronts) {
      num_wavefronts = std::max(2 * num_wavefronts, (size_t)score + 1);
      for (auto& a : arr) a.resize(num_wavefronts, nullptr);
    }
    return has_slot(score);
  }
  Wavefront* get(int c, int32_t score) const { return arr[c][slot(score)]; }
  void set(int c, int32_t score, Wavefront* w) { arr[c][slot(score)] = w; }
};

static inline bool is_null_wf(const Wavefront* w) { return !w || w->null; }
static inline Wavefront* live_or_none(Wavefront* w) { return is_null_wf(w) ? nullptr : w; }
static inline void null_bounds(const Wavefront* w, int32_t& lo, int32_t& hi) {
  if (!w) { lo = 1; hi = -1; } else { lo = w->lo; hi = w->hi; }
}

// ---------------------------------------------------------------------------
// BiWFA breakpoint: src/bialign.rs
// ---------------------------------------------------------------------------
struct Breakpoint {
  int32_t score = INT32_MAX, score_forward = 0, score_reverse = 0;
  int32_t k_forward = 0, k_reverse = 0, offset_forward = 0, offset_reverse = 0;
  int component = CM;
};

enum BiKind { BI_OK, BI_END_REACHED, BI_UNREACHABLE, BI_MAXSTEPS, BI_UNATTAINABLE };
struct BiStatus {
  int kind = BI_OK;
  int32_t score = 0;
};

// scan_overlap + breakpoint_m2m / breakpoint_indel2indel, src/bialign.rs:79-298.
// The SIMD chunking there keeps the ascending-k visiting order; the plain
// ascending scan below visits the same diagonals in the same order.
static void breakpoint_scan(const Wavefront& w0, const Wavefront& w1, int32_t plen, int32_t tlen,
                            int32_t s0, int32_t s1, int32_t gap_opening, int comp, bool indel,
                            bool forward, Breakpoint& bp) {
  if (s0 + s1 - gap_opening >= bp.score) return;
  int32_t lo0 = w0.lo, hi0 = w0.hi;
  int32_t lo1i = (tlen - plen) - w1.hi, hi1i = (tlen - plen) - w1.lo;
  if (hi1i < lo0 || hi0 < lo1i) return;
  int32_t mlo = std::max(lo0, lo1i), mhi = std::min(hi0, hi1i);
  for (int32_t k0 = mlo; k0 <= mhi; ++k0) {
    int32_t k1 = (tlen - plen) - k0;
    int32_t o0 = w0.get(k0), o1 = w1.get(k1);
    if (o0 + o1 < tlen) continue;
    if (indel) {
      int32_t ck = forward ? k0 : k1, ch = forward ? o0 : o1;
      if (ch - ck > plen || ch > tlen) continue;
    }
    if (forward) {
      bp.score_forward = s0; bp.score_reverse = s1; bp.k_forward = k0; bp.k_reverse = k1;
      bp.offset_forward = o0; bp.offset_reverse = o1;
    } else {
      bp.score_forward = s1; bp.score_reverse = s0; bp.k_forward = k1; bp.k_reverse = k0;
      bp.offset_forward = o1; bp.offset_reverse = o0;
    }
    bp.score = s0 + s1 - gap_opening;
    bp.component = comp;
    return;
  }
}

static const Wavefront* valid_wf(const Wavefront* w) { return (w && !w->null) ? w : nullptr; }

// bialign_overlap, src/bialign.rs:362-508
static void bialign_overlap(const Components& c0, const Components& c1, int32_t s0, int32_t s1,
                            int32_t plen, int32_t tlen, int32_t go1, int32_t go2, bool has_affine,
                            bool has_affine2p, bool forward, Breakpoint& bp) {
  size_t scope = c1.scope;
  const Wavefront* m0 = valid_wf(c0.get(CM, s0));
  if (!m0) return;
  const Wavefront* d1_0 = has_affine ? valid_wf(c0.get(CD1, s0)) : nullptr;
  const Wavefront* i1_0 = has_affine ? valid_wf(c0.get(CI1, s0)) : nullptr;
  const Wavefront* d2_0 = has_affine2p ? valid_wf(c0.get(CD2, s0)) : nullptr;
  const Wavefront* i2_0 = has_affine2p ? valid_wf(c0.get(CI2, s0)) : nullptr;
  for (size_t i = 0; i < scope; ++i) {
    int32_t si = s1 - (int32_t)i;
    if (si < 0) break;
    if (has_affine2p && s0 + si - go2 < bp.score) {
      const Wavefront* w;
      if (d2_0 && (w = valid_wf(c1.get(CD2, si))))
        breakpoint_scan(*d2_0, *w, plen, tlen, s0, si, go2, CD2, true, forward, bp);
      if (i2_0 && (w = valid_wf(c1.get(CI2, si))))
        breakpoint_scan(*i2_0, *w, plen, tlen, s0, si, go2, CI2, true, forward, bp);
    }
    if (has_affine && s0 + si - go1 < bp.score) {
      const Wavefront* w;
      if (d1_0 && (w = valid_wf(c1.get(CD1, si))))
        breakpoint_scan(*d1_0, *w, plen, tlen, s0, si, go1, CD1, true, forward, bp);
      if (i1_0 && (w = valid_wf(c1.get(CI1, si))))
        breakpoint_scan(*i1_0, *w, plen, tlen, s0, si, go1, CI1, true, forward, bp);
    }
    if (s0 + si >= bp.score) continue;
    if (const Wavefront* w = valid_wf(c1.get(CM, si)))
      breakpoint_scan(*m0, *w, plen, tlen, s0, si, 0, CM, false, forward, bp);
  }
}

// ---------------------------------------------------------------------------
// Aligner: src/aligner.rs
// ---------------------------------------------------------------------------
enum Span { SPAN_END2END = 0, SPAN_ENDSFREE = 1 };
enum Scope { SCOPE_SCORE = 0, SCOPE_ALIGNMENT = 1 };

struct Pos {
  int32_t score = 0, k = 0, offset = 0;
};

struct Counters {
  int64_t cells = 0, bases = 0, ops = 0;
};

static constexpr int32_t BIALIGN_FALLBACK_MIN_SCORE = 250;   // src/bialign.rs:511
static constexpr int32_t BIALIGN_FALLBACK_MIN_LENGTH = 100;  // src/bialign.rs:515
static constexpr int32_t BIALIGN_RECOVERY_MIN_SCORE = 500;   // src/bialign.rs:520

class Aligner {
 public:
  Sequences seq;
  Components comps;
  std::vector<std::unique_ptr<Wavefront>> pool;
  std::vector<Wavefront*> free_list;
  Penalties pen;
  int scope = SCOPE_SCORE;
  int span = SPAN_END2END;
  Cigar cigar;
  Pos end_pos;
  int status = OK;
  int32_t num_null_steps = 0;
  int32_t p0 = 0, pf = 0, t0 = 0, tf = 0;
  bool extension = false;
  Heuristic heur;
  HeurState hstate;
  int memory_mode = 0;
  bool piggyback = false;  // med/low memory with an alignment (the piggyback backtrace)
  // Med/low run either as the reference does (bt_literal: every cell carries
  // its packed CIGAR and block index, offloaded to `bt`) or by re-making the
  // kernels' picks from the kept offsets after the end cell is found
  // (backtrace_piggyback_rederived); both give the same CIGARs.
  bool bt_literal = true;
  BtBuffer bt;
  uint32_t zdrop_bt_pc = 0, zdrop_bt_pv = BT_BLOCK_IDX_NULL;  // zdrop_best_bt, :186
  bool lit() const { return piggyback && bt_literal; }
  // Compat (src/aligner.rs:53-94): 0 C (reproduce C's known bugs), 1 Corrected.
  int compat = 0;
  // Corrected-mode ends-free end candidate (EndsfreeCandidate, :96-107): the
  // best cell reaching a free end so far and its total score.
  struct Candidate {
    bool has = false;
    int32_t total = 0;
    Pos pos;
    uint32_t bt_pc = 0, bt_pv = BT_BLOCK_IDX_NULL;  // its cell's backtrace (med/low)
  };
  Candidate best;
  // Corrected-mode begin-free dominance pruning (:172-186): per component,
  // the furthest offset each diagonal reached at an earlier score.
  std::vector<int32_t> dom_best;
  int32_t dom_base = 0, dom_len = 0;
  int32_t max_steps = INT32_MAX;
  std::vector<int32_t> scratch;
  Counters ctr;
  std::unique_ptr<Aligner> bi_fwd, bi_rev, bi_base;

  // WavefrontAligner::new, src/aligner.rs:409-459 (components sized for
  // PATTERN_LENGTH_INIT x TEXT_LENGTH_INIT = 1000 x 1000, :377-378).
  explicit Aligner(const Penalties& p) : pen(p) { comps.create(1000, 1000, pen, false); }

  // --- wavefront pool (the slab's role; contents are not semantic) -------
  Wavefront* allocate(int32_t lo, int32_t hi) {
    int32_t len = hi - lo + 1;
    Wavefront* w;
    if (!free_list.empty() && free_list.back()->alloc >= len) {
      w = free_list.back();
      free_list.pop_back();
    } else {
      pool.emplace_back(new Wavefront());
      w = pool.back().get();
      w->reallocate(len);
    }
    if (lit()) w->ensure_bt();
    w->init(lo, hi);
    return w;
  }
  void free_wf(Wavefront* w) { if (w) free_list.push_back(w); }
  void pool_reset() {
    free_list.clear();
    for (auto& w : pool) free_list.push_back(w.get());
    std::sort(free_list.begin(), free_list.end(),
              [](Wavefront* a, Wavefront* b) { return a->alloc < b->alloc; });
  }

  int32_t plen() const { return seq.plen; }
  int32_t tlen() const { return seq.tlen; }

  // endsfree_begin_k, src/aligner.rs:3408-3421
  bool endsfree_begin_k(int32_t score, int32_t& k) const {
    int32_t m = pen.match_;
    if (m == 0 || span != SPAN_ENDSFREE) return false;
    if (t0 == 0 && p0 == 0) return false;
    if (score % (-m) != 0) return false;
    k = score / (-m);
    return t0 >= k || p0 >= k;
  }

  // output_alloc_range, src/aligner.rs:3325-3341
  void output_alloc_range(int32_t score, int32_t lo, int32_t hi, int32_t& alo, int32_t& ahi) {
    int32_t k;
    if (span == SPAN_ENDSFREE && score >= 0 && endsfree_begin_k(score, k)) {
      lo = std::min(lo, -k);
      hi = std::max(hi, k);
    }
    int32_t pad = (int32_t)comps.scope + 1;
    if (lo - pad < comps.alloc_lo || hi + pad > comps.alloc_hi) {
      comps.alloc_lo = std::min(comps.alloc_lo, lo - pad);
      comps.alloc_hi = std::max(comps.alloc_hi, hi + pad);
      comps.resize_null_victim(comps.alloc_lo, comps.alloc_hi);
    }
    alo = comps.alloc_lo;
    ahi = comps.alloc_hi;
  }

  // reuse_or_allocate, src/aligner.rs:3347-3369
  Wavefront* reuse_or_allocate(Wavefront* old, int32_t alo, int32_t ahi) {
    if (old) {
      if (old->alloc >= ahi - alo + 1) {
        old->init(alo, ahi);
        return old;
      }
      free_wf(old);
    }
    return allocate(alo, ahi);
  }

  // The seed's backtrace starts at (v, h) = (offset - k, offset) (set_bt_init,
  // src/aligner.rs:213-225, and :3425-3434).
  void endsfree_init_offset(Wavefront& wf, int32_t k, int32_t v, int32_t h) {
    wf.set(k, h);
    if (piggyback) { wf.seeds.push_back(k); wf.mark_written(k, k); }
    if (lit()) set_bt_init(wf, k, v, h);
  }
  // set_bt_init, src/aligner.rs:213-225: an empty pcigar continuing a new
  // initial block at (v, h).
  void set_bt_init(Wavefront& wf, int32_t k, int32_t v, int32_t h) { wf.set_bt(k, 0, bt.init_block(v, h)); }

  // endsfree_init, src/aligner.rs:3426-3452
  void endsfree_init(Wavefront& wf, int32_t k) {
    int32_t lo = wf.lo, hi = wf.hi;
    if (t0 >= k) {
      if (hi >= k) {
        if (wf.get(k) <= k) endsfree_init_offset(wf, k, 0, k);
      } else {
        for (int32_t kk = hi + 1; kk < k; ++kk) wf.set(kk, OFFSET_NULL);
        endsfree_init_offset(wf, k, 0, k);
        wf.hi = k;
      }
    }
    if (p0 >= k) {
      if (lo <= -k) {
        if (wf.get(-k) <= 0) endsfree_init_offset(wf, -k, k, 0);
      } else {
        endsfree_init_offset(wf, -k, k, 0);
        for (int32_t kk = -k + 1; kk < lo; ++kk) wf.set(kk, OFFSET_NULL);
        wf.lo = -k;
      }
    }
  }

  // endsfree_null_m, src/aligner.rs:3470-3494
  Wavefront* endsfree_null_m(int32_t k) {
    bool text = t0 >= k, pattern = p0 >= k;
    int32_t lo, hi;
    if (text && pattern) { lo = -k; hi = k; }
    else if (text) { lo = k; hi = k; }
    else if (pattern) { lo = -k; hi = -k; }
    else { lo = 0; hi = 0; }
    int32_t alo, ahi;
    output_alloc_range(-1, lo, hi, alo, ahi);
    Wavefront* wf = allocate(alo, ahi);
    for (int32_t kk = lo; kk <= hi; ++kk) wf->set(kk, OFFSET_NULL);
    if (text) endsfree_init_offset(*wf, k, 0, k);
    if (pattern) endsfree_init_offset(*wf, -k, k, 0);
    wf->set_limits(lo, hi);
    return wf;
  }

  void set_null_output(int32_t score, int ncomp) {  // :3498-3530
    size_t s = comps.slot(score);
    for (int c = 0; c < ncomp; ++c) {
      if (comps.modular) free_wf(comps.arr[c][s]);
      comps.arr[c][s] = nullptr;
    }
  }

  int ncomp() const { return pen.metric == AFFINE ? 3 : pen.metric == AFFINE2P ? 5 : 1; }

  void clamp_to_band(int32_t& lo, int32_t& hi) const {  // :3308-3317
    if (heur.banded()) { lo = std::max(lo, heur.p0); hi = std::min(hi, heur.p1); }
  }

  // --- init_alignment, src/aligner.rs:846-1000 ---------------------------
  void init_alignment() {
    int32_t n = plen(), m = tlen();
    if (scope == SCOPE_ALIGNMENT) cigar.resize((size_t)(2 * (n + m)) + 1);
    bool score_only = scope == SCOPE_SCORE;
    // Med/low with an alignment: the piggyback backtrace.  Its CIGAR is the
    // chain of operations each cell copies from the predecessor its kernel
    // picked (src/compute/piggyback.rs), so the oracle keeps every score
    // (no score cap, as the reference's modular components have none) and
    // walks those choices back from the end cell (backtrace_piggyback).
    piggyback = !score_only && memory_mode != 0;
    comps.modular = score_only;
    comps.grow = piggyback;
    comps.resize(n, m, pen);
    pool_reset();
    num_null_steps = 0;
    status = OK;
    end_pos = Pos{-1, DIAG_NULL, OFFSET_NULL};
    hstate.reset(heur);
    int32_t sc = (int32_t)comps.scope;
    comps.hist_lo = -(n + sc + 2);
    comps.hist_hi = m + sc + 2;
    // Corrected mode (:912-947): no candidate yet; dominance pruning only
    // with begin-free seeds (at most 4 bases unless gap-linear) and no
    // heuristic that reads the wavefronts.
    best = Candidate();
    dom_best.clear();
    const int32_t bfree = std::max(p0, t0);
    if (endsfree_corrected() && span == SPAN_ENDSFREE && bfree > 0 &&
        (pen.metric == LINEAR || bfree <= 4) &&
        (heur.kind == H_NONE || heur.kind == H_BANDED_STATIC)) {
      dom_base = comps.hist_lo;
      dom_len = comps.hist_hi - comps.hist_lo + 1;
      dom_best.assign((size_t)ncomp() * (size_t)dom_len, -1);
    }
    int32_t lo0 = 0, hi0 = 0;
    if (pen.match_ == 0 && span == SPAN_ENDSFREE) { lo0 = -p0; hi0 = t0; }
    int32_t alo, ahi;
    output_alloc_range(0, lo0, hi0, alo, ahi);
    if (lit()) {
      bt.clear();
      comps.null_wf.ensure_bt();
      zdrop_bt_pc = 0;
      zdrop_bt_pv = BT_BLOCK_IDX_NULL;
    }
    Wavefront* wf = allocate(alo, ahi);
    wf->set(0, 0);
    wf->set_limits(0, 0);
    if (lit()) set_bt_init(*wf, 0, 0, 0);
    if (span == SPAN_ENDSFREE && pen.match_ == 0) {
      for (int32_t h = 1; h <= t0; ++h) {
        wf->set(h, h);
        if (lit()) set_bt_init(*wf, h, 0, h);
      }
      for (int32_t v = 1; v <= p0; ++v) {
        wf->set(-v, 0);
        if (lit()) set_bt_init(*wf, -v, v, 0);
      }
      wf->lo = -p0; wf->hi = t0; wf->init_min = -p0; wf->init_max = t0;
      if (piggyback) wf->mark_written(-p0, t0);
    }
    comps.set(CM, 0, wf);
    ctr = Counters();
  }

  // init_alignment_component, src/aligner.rs:3205-3265
  void init_alignment_component(int comp) {
    int32_t n = plen(), m = tlen();
    if (scope == SCOPE_ALIGNMENT) cigar.resize((size_t)(2 * (n + m)) + 1);
    comps.resize(n, m, pen);
    pool_reset();
    num_null_steps = 0;
    status = OK;
    end_pos = Pos{0, 0, 0};
    hstate.reset(heur);
    int32_t sc = (int32_t)comps.scope;
    comps.hist_lo = -(n + sc + 2);
    comps.hist_hi = m + sc + 2;
    int32_t alo, ahi;
    output_alloc_range(0, 0, 0, alo, ahi);
    Wavefront* wf = allocate(alo, ahi);
    wf->set(0, 0);
    wf->set_limits(0, 0);
    comps.set(comp, 0, wf);
  }

  // --- extend: src/extend.rs:15-177 ----------------------------------------
  int32_t extend_one(int32_t k, int32_t off) {
    const uint8_t* P = seq.P();
    const uint8_t* T = seq.T();
    int64_t v = off - k, h = off;
    int64_t pmax = (int64_t)(seq.buf.size() - seq.pstart), tmax = (int64_t)(seq.buf.size() - seq.tstart);
    int32_t start = off;
    while (v < pmax && h < tmax && P[v] == T[h]) { ++v; ++h; ++off; }
    ctr.bases += (off - start) + 1;
    return off;
  }
  void extend_end2end_wf(Wavefront& wf) {  // extend_matches_packed_end2end :47
    for (int32_t k = wf.lo; k <= wf.hi; ++k) {
      int32_t off = wf.get(k);
      if (off >= 0) wf.set(k, extend_one(k, off));
    }
  }
  int32_t extend_end2end_max_wf(Wavefront& wf) {  // _end2end_max :73
    int32_t mx = 0;
    for (int32_t k = wf.lo; k <= wf.hi; ++k) {
      int32_t off = wf.get(k);
      if (off >= 0) {
        int32_t e = extend_one(k, off);
        wf.set(k, e);
        if (2 * e - k > mx) mx = 2 * e - k;
      }
    }
    return mx;
  }
  // termination_endsfree, src/termination.rs:31-58
  bool term_endsfree(int32_t k, int32_t off) const {
    int32_t h = off, v = off - k;
    if (h >= tlen() && plen() - v <= pf) return true;
    if (v >= plen() && tlen() - h <= tf) return true;
    return false;
  }
  bool extend_endsfree_wf(Wavefront& wf, int32_t& rk, int32_t& roff) {  // _endsfree :112
    for (int32_t k = wf.lo; k <= wf.hi; ++k) {
      int32_t off = wf.get(k);
      if (off != OFFSET_NULL) {
        off = extend_one(k, off);
        wf.set(k, off);
        if (term_endsfree(k, off)) { rk = k; roff = off; return true; }
      }
    }
    return false;
  }

  DropParams drop_params() const {  // :1391 + DropParams::new
    DropParams d;
    bool endsfree = span == SPAN_ENDSFREE;
    bool bf = pen.match_ == 0 && endsfree;
    d.swg_match = pen.match_ != 0 ? -pen.match_ : 1;
    d.pattern_begin_free = bf ? p0 : 0;
    d.text_begin_free = bf ? t0 : 0;
    d.max_penalty = (int32_t)comps.scope - 1;
    return d;
  }

  // apply_heuristic_cutoff, src/aligner.rs:1644-1766
  bool apply_heuristic_cutoff(int32_t score, Wavefront* m) {
    if (heur.kind == H_BANDED_STATIC && m->lo >= heur.p0 && m->hi <= heur.p1) return false;
    DropParams drop = drop_params();
    int32_t sbase = comps.alloc_lo - 2;
    size_t need = (size_t)(comps.alloc_hi + 2 - sbase + 1);
    if (scratch.size() < need) scratch.assign(need, 0);
    int32_t lo_base = m->lo, hi_base = m->hi;
    const int32_t max_wf_score_base = hstate.max_wf_score;
    bool z = heuristic_cutoff(heur, hstate, *m, scratch, sbase, plen(), tlen(), drop, score);
    // Corrected med/low keep the backtrace of a new Z-drop best cell, which
    // the end backtrace needs after its wavefront is gone (:1677-1688).
    if (compat == 1 && lit() && hstate.max_wf_score == score && max_wf_score_base != score)
      m->bt_or_zero(hstate.max_sw_score_k, zdrop_bt_pc, zdrop_bt_pv);
    if (z) {
      end_pos = Pos{hstate.max_wf_score, hstate.max_sw_score_k, hstate.max_sw_score_offset};
      return true;
    }
    if (lo_base > hi_base || (m->lo == lo_base && m->hi == hi_base)) return false;
    if (m->lo > m->hi) { m->null = true; m->clear_init_range(); }
    if (pen.metric == AFFINE || pen.metric == AFFINE2P) {
      int cs[4] = {CI1, CD1, CI2, CD2};
      int nc = pen.metric == AFFINE ? 2 : 4;
      for (int i = 0; i < nc; ++i) {
        Wavefront* w = comps.get(cs[i], score);
        if (!w) continue;
        if (m->lo > w->lo) w->lo = m->lo;
        if (m->hi < w->hi) w->hi = m->hi;
        if (w->lo > w->hi) { w->null = true; w->clear_init_range(); }
      }
    }
    return false;
  }

  // extend_end2end, src/aligner.rs:1004-1050
  bool extend_end2end(int32_t score) {
    Wavefront* m = comps.get(CM, score);
    if (!m) {
      if (num_null_steps > (int32_t)comps.scope) { status = END_UNREACHABLE; return true; }
      return false;
    }
    extend_end2end_wf(*m);
    int32_t ak = tlen() - plen();
    if (!(m->lo > ak || ak > m->hi) && m->get(ak) >= tlen()) {  // termination_end2end
      end_pos = Pos{score, ak, tlen()};
      status = END_REACHED;
      return true;
    }
    if (heur.kind != H_NONE && apply_heuristic_cutoff(score, m)) {
      status = END_UNREACHABLE;
      return true;
    }
    return false;
  }

  // extend_endsfree, src/aligner.rs:1053-1101 (C compatibility)
  bool extend_endsfree(int32_t score) {
    if (endsfree_corrected()) return extend_endsfree_corrected(score);
    Wavefront* m = comps.get(CM, score);
    if (!m) {
      if (num_null_steps > (int32_t)comps.scope) { status = END_UNREACHABLE; return true; }
      return false;
    }
    int32_t k, off;
    if (extend_endsfree_wf(*m, k, off)) {
      end_pos = Pos{score, k, off};
      status = END_REACHED;
      return true;
    }
    if (heur.kind != H_NONE && apply_heuristic_cutoff(score, m)) {
      status = END_UNREACHABLE;
      return true;
    }
    return false;
  }

  // --- Compat::Corrected ends-free (src/aligner.rs:1104-1345) ----------------
  bool endsfree_corrected() const { return compat == 1 && pen.match_ < 0; }  // :1107

  // endsfree_left, src/termination.rs:65-86: the bases a cell at a free end
  // leaves to the free end gap (the smaller of the two ends it reaches).
  bool endsfree_left(int32_t k, int32_t off, int32_t& left) const {
    const int32_t n = plen(), m = tlen(), h = off, v = off - k;
    const bool by_t = h >= m && n - v <= pf, by_p = v >= n && m - h <= tf;
    if (!by_t && !by_p) return false;
    left = by_t && by_p ? std::min(n - v, m - h) : by_t ? n - v : m - h;
    return true;
  }
  // extend_matches_packed_endsfree_best, src/extend.rs:179-232: extend every
  // cell (no early stop) and return the free-end cell leaving the fewest
  // bases (the lowest diagonal on ties).
  bool extend_endsfree_best_wf(Wavefront& wf, int32_t& rk, int32_t& roff, int32_t& rleft) {
    bool found = false;
    for (int32_t k = wf.lo; k <= wf.hi; ++k) {
      int32_t off = wf.get(k);
      if (off == OFFSET_NULL) continue;
      off = extend_one(k, off);
      wf.set(k, off);
      int32_t left;
      if (term_endsfree(k, off) && endsfree_left(k, off, left) && (!found || left < rleft)) {
        found = true; rk = k; roff = off; rleft = left;
      }
    }
    return found;
  }
  // Wavefront::trim_nulled, src/wavefront.rs:463-490
  static void trim_nulled(Wavefront& wf, int32_t lo, int32_t hi) {
    if (wf.null || wf.lo > wf.hi || (lo <= wf.lo && hi >= wf.hi)) return;
    const int32_t olo = wf.lo, ohi = wf.hi;
    const int32_t nlo = std::max(lo, olo), nhi = std::min(hi, ohi);
    if (nlo > nhi) {
      for (int32_t k = olo; k <= ohi; ++k) wf.set(k, OFFSET_NULL);
      wf.null = true;
    } else {
      for (int32_t k = olo; k < nlo; ++k) wf.set(k, OFFSET_NULL);
      for (int32_t k = nhi + 1; k <= ohi; ++k) wf.set(k, OFFSET_NULL);
    }
    wf.lo = nlo;
    wf.hi = nhi;
  }
  // endsfree_prune, :1214-1255: null the diagonals farther than
  // (total - score) / -match from the end diagonal, in every component.
  void endsfree_prune(int32_t score, int32_t total) {
    const int32_t radius = (total - score) / -pen.match_;
    const int32_t kend = tlen() - plen();
    for (int c = 0; c < ncomp(); ++c) {
      Wavefront* w = comps.get(c, score);
      if (w) trim_nulled(*w, kend - radius, kend + radius);
    }
  }
  // endsfree_dominance_prune, :1257-1320: trim from the ends the cells of a
  // just-computed component that reach no further than a cell of that
  // component did at an earlier score; with `record`, keep the kept offsets.
  void dominance_prune(Wavefront& wf, int c, bool record) {
    if (wf.lo > wf.hi) return;
    const int32_t lo = wf.lo, n = wf.hi - wf.lo + 1;
    int32_t* b = &dom_best[(size_t)c * dom_len + (size_t)(lo - dom_base)];
    int32_t first = 0, last = n;
    while (first < n && wf.get(lo + first) <= b[first]) ++first;
    while (last > first && wf.get(lo + last - 1) <= b[last - 1]) --last;
    if (record)
      for (int32_t i = first; i < last; ++i) b[i] = std::max(b[i], wf.get(lo + i));
    for (int32_t i = 0; i < first; ++i) wf.set(lo + i, OFFSET_NULL);
    for (int32_t i = last; i < n; ++i) wf.set(lo + i, OFFSET_NULL);
    if (first == last) { wf.lo = 1; wf.hi = 0; wf.null = true; }
    else { wf.lo = lo + first; wf.hi = lo + last - 1; }
  }
  // endsfree_dominance_update, :1322-1338 (M, after extend)
  void dominance_update(const Wavefront& wf, int c) {
    if (wf.null || wf.lo > wf.hi) return;
    int32_t* b = &dom_best[(size_t)c * dom_len + (size_t)(wf.lo - dom_base)];
    for (int32_t k = wf.lo; k <= wf.hi; ++k) b[k - wf.lo] = std::max(b[k - wf.lo], wf.get(k));
  }
  // The dominance pruning of a compute step's outputs, after trim_ends
  // (:1999-2001, :2187-2191, :2541-2550): M without recording, the gap
  // components recording their kept offsets.
  void dominance_outputs(int32_t score) {
    if (dom_best.empty()) return;
    for (int c = 0; c < ncomp(); ++c) {
      Wavefront* w = comps.get(c, score);
      if (w) dominance_prune(*w, c, c != CM);
    }
  }
  // extend_endsfree_corrected, :1123-1211
  bool extend_endsfree_corrected(int32_t score) {
    Wavefront* m = comps.get(CM, score);
    const bool prune = heur.kind == H_NONE || heur.kind == H_BANDED_STATIC;
    if (prune && best.has && best.total > score) endsfree_prune(score, best.total);
    if (m) {
      int32_t k, off, left;
      if (extend_endsfree_best_wf(*m, k, off, left)) {
        const int32_t total = score + (-pen.match_) * left;
        if (!best.has || total < best.total) {
          best.has = true;
          best.total = total;
          best.pos = Pos{score, k, off};
          if (lit()) m->bt_or_zero(k, best.bt_pc, best.bt_pv);  // :1155-1160
          if (prune && total > score) endsfree_prune(score, total);
        }
      }
    }
    if (!dom_best.empty() && !is_null_wf(m)) dominance_update(*m, CM);
    if (best.has && best.total <= score) {  // no later cell can beat it
      end_pos = best.pos;
      status = END_REACHED;
      return true;
    }
    bool done;
    if (!m) done = !best.has && num_null_steps > (int32_t)comps.scope;
    else done = heur.kind != H_NONE && apply_heuristic_cutoff(score, m);
    if (done) {
      if (best.has) { end_pos = best.pos; status = END_REACHED; }
      else status = END_UNREACHABLE;
      return true;
    }
    return false;
  }

  // --- the piggyback kernels' per-cell backtraces, src/compute/piggyback.rs --
  // Every cell copies (pcigar, prev) from the input its kernel picked and
  // pushes the operation: edit/linear cells pick misms over del over ins
  // (later checks win ties, :197-228), indel del over ins (:249-273); a gap
  // cell picks its extension over the M opening on a tie (`gap`, :146-170)
  // and affine M picks misms, else D2, D1, I2, I1, pushing an X (the gap
  // close) on the chosen chain (:364-392, 483-527).
  void bt_edit_cells(const Wavefront& wi, const Wavefront& wx, const Wavefront& wd, Wavefront& out,
                     int32_t lo, int32_t hi, bool indel) {
    for (int32_t k = lo; k <= hi; ++k) {
      const int32_t ins = wrap_add(wi.get(k - 1), 1), del = wd.get(k + 1);
      uint32_t pc, pv;
      if (indel) {
        const bool d = std::max(del, ins) == del;
        pc = d ? pcigar_push(wd.get_pc(k + 1), PCIGAR_DELETION) : pcigar_push(wi.get_pc(k - 1), PCIGAR_INSERTION);
        pv = d ? wd.get_pv(k + 1) : wi.get_pv(k - 1);
      } else {
        const int32_t misms = wrap_add(wx.get(k), 1);
        const int32_t mx = std::max(del, std::max(ins, misms));
        const bool d = mx == del, x = mx == misms;
        pc = x ? pcigar_push(wx.get_pc(k), PCIGAR_MISMATCH)
               : d ? pcigar_push(wd.get_pc(k + 1), PCIGAR_DELETION)
                   : pcigar_push(wi.get_pc(k - 1), PCIGAR_INSERTION);
        pv = x ? wx.get_pv(k) : d ? wd.get_pv(k + 1) : wi.get_pv(k - 1);
      }
      out.set_bt(k, pc, pv);
    }
  }
  struct GapPick {
    int32_t off;
    uint32_t pc, pv;
  };
  // `gap` (:146-170): the M opening at kk or the extension at kk, the
  // extension on a tie.
  static GapPick gap_pick(const Wavefront& open, const Wavefront& ext, int32_t kk) {
    const int32_t o = open.get(kk), e = ext.get(kk);
    return e >= o ? GapPick{e, ext.get_pc(kk), ext.get_pv(kk)} : GapPick{o, open.get_pc(kk), open.get_pv(kk)};
  }
  void bt_affine_cells(const Wavefront& wmm, const Wavefront& wo1, const Wavefront& wi1,
                       const Wavefront& wd1, const Wavefront* wo2, const Wavefront* wi2,
                       const Wavefront* wd2, Wavefront& mc, Wavefront& ic, Wavefront& dc,
                       Wavefront* i2c, Wavefront* d2c, int32_t lo, int32_t hi) {
    const bool two = i2c != nullptr;
    for (int32_t k = lo; k <= hi; ++k) {
      GapPick i1 = gap_pick(wo1, wi1, k - 1), d1 = gap_pick(wo1, wd1, k + 1);
      i1.off = wrap_add(i1.off, 1);
      i1.pc = pcigar_push(i1.pc, PCIGAR_INSERTION);
      d1.pc = pcigar_push(d1.pc, PCIGAR_DELETION);
      ic.set_bt(k, i1.pc, i1.pv);
      dc.set_bt(k, d1.pc, d1.pv);
      const int32_t misms = wrap_add(wmm.get(k), 1);
      uint32_t pc, pv;
      int32_t mx;
      if (!two) {
        mx = std::max(d1.off, std::max(misms, i1.off));
        const bool d = mx == d1.off;
        pc = d ? d1.pc : i1.pc;
        pv = d ? d1.pv : i1.pv;
      } else {
        GapPick i2 = gap_pick(*wo2, *wi2, k - 1), d2 = gap_pick(*wo2, *wd2, k + 1);
        i2.off = wrap_add(i2.off, 1);
        i2.pc = pcigar_push(i2.pc, PCIGAR_INSERTION);
        d2.pc = pcigar_push(d2.pc, PCIGAR_DELETION);
        i2c->set_bt(k, i2.pc, i2.pv);
        d2c->set_bt(k, d2.pc, d2.pv);
        mx = std::max(std::max(std::max(i1.off, i2.off), std::max(d1.off, d2.off)), misms);
        const bool s2 = mx == i2.off, t1 = mx == d1.off, t2 = mx == d2.off;
        pc = t2 ? d2.pc : t1 ? d1.pc : s2 ? i2.pc : i1.pc;
        pv = t2 ? d2.pv : t1 ? d1.pv : s2 ? i2.pv : i1.pv;
      }
      const bool x = mx == misms;
      mc.set_bt(k, pcigar_push(x ? wmm.get_pc(k) : pc, PCIGAR_MISMATCH), x ? wmm.get_pv(k) : pv);
    }
  }

  // --- offloading, C's wavefront_backtrace_offload.c (piggyback.rs:530-705) --
  // Every live cell's pcigar at or above `mask` moves into a new block, the
  // cell continuing from it.
  void offload_selective(Wavefront& wf, int32_t lo, int32_t hi, uint32_t mask) {
    for (int32_t k = lo; k <= hi; ++k) {
      const uint32_t pc = wf.get_pc(k);
      if (wf.get(k) >= 0 && pc >= mask) wf.set_bt(k, 0, bt.store_block(pc, wf.get_pv(k)));
    }
  }
  int32_t offload_blocks_linear(Wavefront& wf, int32_t lo, int32_t hi) {  // :557-569
    const bool low = memory_mode == 2;
    offload_selective(wf, lo, hi, low ? PCIGAR_FULL_MASK : PCIGAR_HALF_FULL_MASK);
    return low ? PCIGAR_MAX_LENGTH - 1 : PCIGAR_MAX_LENGTH / 2;
  }
  int32_t offload_blocks_affine(Wavefront& wf, int32_t lo, int32_t hi) {  // :573-585
    const bool low = memory_mode == 2;
    offload_selective(wf, lo, hi, low ? PCIGAR_ALMOST_FULL_MASK : PCIGAR_HALF_FULL_MASK);
    return low ? PCIGAR_MAX_LENGTH - 2 : PCIGAR_MAX_LENGTH / 2;
  }
  static int32_t occ_of(const Wavefront* w) { return is_null_wf(w) ? 0 : w->occ; }
  static int32_t occ_gap(const Wavefront* open, const Wavefront* ext) {  // :611-620
    int32_t o = is_null_wf(open) ? 0 : open->occ + 1;
    if (!is_null_wf(ext)) o = std::max(o, ext->occ + 1);
    return o;
  }
  void offload_component(Wavefront* wf, int32_t lo, int32_t hi) {  // :622-632
    if (wf && !wf->null && wf->occ >= PCIGAR_MAX_LENGTH - 1) wf->occ = offload_blocks_affine(*wf, lo, hi);
  }

  // --- compute steps --------------------------------------------------------
  // compute_edit_step, src/aligner.rs:1769-1864 (+ compute_edit_idm /
  // compute_indel_idm, src/compute/edit.rs:16-233)
  void compute_edit_step(int32_t score) {
    Wavefront* prev = comps.get(CM, score - 1);
    if (is_null_wf(prev)) { ++num_null_steps; set_null_output(score, 1); return; }
    num_null_steps = 0;
    int32_t plo = prev->lo, phi = prev->hi;
    int32_t lo = std::max(plo - 1, comps.hist_lo + 1);
    int32_t hi = std::min(phi + 1, comps.hist_hi - 1);
    if (lo > hi) { set_null_output(score, 1); return; }
    for (int32_t k : {plo - 2, plo - 1, phi + 1, phi + 2}) prev->set_null_cell_if_allocated(k);
    int32_t alo, ahi;
    output_alloc_range(score, lo, hi, alo, ahi);
    Wavefront* old = comps.modular ? comps.get(CM, score) : nullptr;
    Wavefront* cur = reuse_or_allocate(old, alo, ahi);
    cur->set_limits(lo, hi);
    ctr.cells += hi - lo + 1;
    bool indel = pen.metric == INDEL;
    int32_t n = plen(), m = tlen();
    for (int32_t k = lo; k <= hi; ++k) {
      int32_t ins = prev->get(k - 1), del = prev->get(k + 1), mx;
      if (indel) mx = std::max(del, ins + 1);
      else mx = std::max(del, std::max(ins, prev->get(k)) + 1);
      if ((uint32_t)mx > (uint32_t)m || (uint32_t)(mx - k) > (uint32_t)n) mx = OFFSET_NULL;
      cur->set(k, mx);
    }
    if (lit()) {
      bt_edit_cells(*prev, *prev, *prev, *cur, lo, hi, indel);
      // C offloads edit/indel every PCIGAR_MAX_LENGTH scores (:1848-1852).
      if (score % PCIGAR_MAX_LENGTH == 0) offload_blocks_linear(*cur, lo, hi);
    }
    comps.set(CM, score, cur);
    trim_ends(n, m, *cur);
    dominance_outputs(score);
  }

  // compute_linear_step, src/aligner.rs:1867-2003 (+ compute_linear_idm,
  // src/compute/linear.rs:21-133)
  void compute_linear_step(int32_t score) {
    int32_t ms = score - pen.mismatch, gs = score - pen.o1;
    Wavefront* misms = ms >= 0 ? comps.get(CM, ms) : nullptr;
    Wavefront* gap = gs >= 0 ? comps.get(CM, gs) : nullptr;
    int32_t bk;
    if (is_null_wf(misms) && is_null_wf(gap)) {
      ++num_null_steps;
      set_null_output(score, 1);
      if (endsfree_begin_k(score, bk)) comps.set(CM, score, endsfree_null_m(bk));
      return;
    }
    num_null_steps = 0;
    misms = live_or_none(misms);
    gap = live_or_none(gap);
    int32_t mlo, mhi, glo, ghi;
    null_bounds(misms, mlo, mhi);
    null_bounds(gap, glo, ghi);
    int32_t lo = std::min(mlo, glo - 1), hi = std::max(mhi, ghi + 1);
    clamp_to_band(lo, hi);
    lo = std::max(lo, comps.hist_lo + 1);
    hi = std::min(hi, comps.hist_hi - 1);
    if (lo > hi) { set_null_output(score, 1); return; }
    int32_t alo, ahi;
    output_alloc_range(score, lo, hi, alo, ahi);
    if (misms) { misms->init_ends_higher(hi); misms->init_ends_lower(lo); }
    if (gap) { gap->init_ends_higher(hi + 1); gap->init_ends_lower(lo - 1); }
    Wavefront* old = comps.modular ? comps.get(CM, score) : nullptr;
    Wavefront* cur = reuse_or_allocate(old, alo, ahi);
    cur->set_limits(lo, hi);
    ctr.cells += hi - lo + 1;
    const Wavefront& wm = misms ? *misms : comps.null_wf;
    const Wavefront& wg = gap ? *gap : comps.null_wf;
    int32_t n = plen(), m = tlen();
    for (int32_t k = lo; k <= hi; ++k) {
      int32_t mi = wm.get(k) + 1, ins = wg.get(k - 1) + 1, del = wg.get(k + 1);
      int32_t mx = std::max(del, std::max(ins, mi));
      if ((uint32_t)mx > (uint32_t)m || (uint32_t)(mx - k) > (uint32_t)n) mx = OFFSET_NULL;
      cur->set(k, mx);
    }
    if (lit()) {
      bt_edit_cells(wg, wm, wg, *cur, lo, hi, false);
      // offload_linear (:590-607)
      cur->occ = std::max(occ_of(gap), occ_of(misms)) + 1;
      if (!cur->null && cur->occ >= PCIGAR_MAX_LENGTH) cur->occ = offload_blocks_linear(*cur, lo, hi);
    }
    comps.set(CM, score, cur);
    if (endsfree_begin_k(score, bk)) endsfree_init(*cur, bk);
    trim_ends(n, m, *cur);
    dominance_outputs(score);
  }

  // compute_affine_step, src/aligner.rs:2006-2193 and compute_affine2p_step,
  // :2201-2553 (+ compute_affine_idm, src/compute/affine.rs:28-351, and
  // compute_affine2p_idm, src/compute/affine2p.rs:32-235).  One routine:
  // affine is the two-piece step with the second piece absent.
  void compute_affine_step(int32_t score) {
    const bool two = pen.metric == AFFINE2P;
    int32_t x = pen.mismatch, oe1 = pen.o1 + pen.e1, e1 = pen.e1;
    int32_t oe2 = pen.o2 + pen.e2, e2 = pen.e2;
    size_t out = comps.slot(score);
    Wavefront* m_misms = score - x >= 0 ? comps.get(CM, score - x) : nullptr;
    Wavefront* m_open1 = score - oe1 >= 0 ? comps.get(CM, score - oe1) : nullptr;
    Wavefront* m_open2 = (two && score - oe2 >= 0) ? comps.get(CM, score - oe2) : nullptr;
    Wavefront *i1e = nullptr, *d1e = nullptr, *i2e = nullptr, *d2e = nullptr;
    if (score - e1 >= 0) { i1e = comps.get(CI1, score - e1); d1e = comps.get(CD1, score - e1); }
    if (two && score - e2 >= 0) { i2e = comps.get(CI2, score - e2); d2e = comps.get(CD2, score - e2); }
    int nc = two ? 5 : 3;
    int32_t bk;
    if (is_null_wf(m_misms) && is_null_wf(m_open1) && is_null_wf(m_open2) && is_null_wf(i1e) &&
        is_null_wf(d1e) && is_null_wf(i2e) && is_null_wf(d2e)) {
      ++num_null_steps;
      set_null_output(score, nc);
      if (endsfree_begin_k(score, bk)) comps.arr[CM][out] = endsfree_null_m(bk);
      return;
    }
    num_null_steps = 0;
    m_misms = live_or_none(m_misms); m_open1 = live_or_none(m_open1); m_open2 = live_or_none(m_open2);
    i1e = live_or_none(i1e); d1e = live_or_none(d1e); i2e = live_or_none(i2e); d2e = live_or_none(d2e);
    bool i2_active = m_open2 || i2e, d2_active = m_open2 || d2e;
    bool affine_kernel = !two || (!i2_active && !d2_active);
    int32_t a, b, lo, hi;
    null_bounds(m_misms, a, b); lo = a; hi = b;
    null_bounds(m_open1, a, b); lo = std::min(lo, a - 1); hi = std::max(hi, b + 1);
    if (two) { null_bounds(m_open2, a, b); lo = std::min(lo, a - 1); hi = std::max(hi, b + 1); }
    null_bounds(i1e, a, b); lo = std::min(lo, a + 1); hi = std::max(hi, b + 1);
    if (two) { null_bounds(i2e, a, b); lo = std::min(lo, a + 1); hi = std::max(hi, b + 1); }
    null_bounds(d1e, a, b); lo = std::min(lo, a - 1); hi = std::max(hi, b - 1);
    if (two) { null_bounds(d2e, a, b); lo = std::min(lo, a - 1); hi = std::max(hi, b - 1); }
    clamp_to_band(lo, hi);
    if (lo > hi) { if (comps.modular) set_null_output(score, nc); return; }
    lo = std::max(lo, comps.hist_lo + 1);
    hi = std::min(hi, comps.hist_hi - 1);
    if (lo > hi) { if (comps.modular) set_null_output(score, nc); return; }
    int32_t alo, ahi;
    output_alloc_range(score, lo, hi, alo, ahi);
    if (m_misms) { m_misms->init_ends_higher(hi); m_misms->init_ends_lower(lo); }
    if (m_open1) { m_open1->init_ends_higher(hi + 1); m_open1->init_ends_lower(lo - 1); }
    if (m_open2) { m_open2->init_ends_higher(hi + 1); m_open2->init_ends_lower(lo - 1); }
    if (i1e) { i1e->init_ends_higher(hi); i1e->init_ends_lower(lo - 1); }
    if (i2e) { i2e->init_ends_higher(hi); i2e->init_ends_lower(lo - 1); }
    if (d1e) { d1e->init_ends_higher(hi + 1); d1e->init_ends_lower(lo); }
    if (d2e) { d2e->init_ends_higher(hi + 1); d2e->init_ends_lower(lo); }
    Wavefront *mc, *ic, *dc, *i2c = nullptr, *d2c = nullptr;
    if (comps.modular) {
      mc = reuse_or_allocate(comps.arr[CM][out], alo, ahi);
      ic = reuse_or_allocate(comps.arr[CI1][out], alo, ahi);
      dc = reuse_or_allocate(comps.arr[CD1][out], alo, ahi);
    } else {
      mc = allocate(alo, ahi); ic = allocate(alo, ahi); dc = allocate(alo, ahi);
    }
    if (two && !affine_kernel) {
      if (comps.modular) {
        i2c = reuse_or_allocate(comps.arr[CI2][out], alo, ahi);
        d2c = reuse_or_allocate(comps.arr[CD2][out], alo, ahi);
      } else {
        i2c = allocate(alo, ahi); d2c = allocate(alo, ahi);
      }
    }
    mc->set_limits(lo, hi); ic->set_limits(lo, hi); dc->set_limits(lo, hi);
    if (i2c) { i2c->set_limits(lo, hi); d2c->set_limits(lo, hi); }
    ctr.cells += hi - lo + 1;
    const Wavefront& NW = comps.null_wf;
    const Wavefront& wmm = m_misms ? *m_misms : NW;
    const Wavefront& wo1 = m_open1 ? *m_open1 : NW;
    const Wavefront& wo2 = m_open2 ? *m_open2 : NW;
    const Wavefront& wi1 = i1e ? *i1e : NW;
    const Wavefront& wd1 = d1e ? *d1e : NW;
    const Wavefront& wi2 = i2e ? *i2e : NW;
    const Wavefront& wd2 = d2e ? *d2e : NW;
    int32_t n = plen(), m = tlen();
    for (int32_t k = lo; k <= hi; ++k) {
      int32_t i1 = std::max(wo1.get(k - 1), wi1.get(k - 1)) + 1;
      int32_t d1 = std::max(wo1.get(k + 1), wd1.get(k + 1));
      int32_t mi = wmm.get(k) + 1;
      int32_t mx;
      if (affine_kernel) {
        mx = std::max(mi, std::max(i1, d1));
      } else {
        int32_t i2 = std::max(wo2.get(k - 1), wi2.get(k - 1)) + 1;
        int32_t d2 = std::max(wo2.get(k + 1), wd2.get(k + 1));
        mx = std::max(mi, std::max(std::max(i1, i2), std::max(d1, d2)));
        i2c->set(k, i2);
        d2c->set(k, d2);
      }
      if ((uint32_t)mx > (uint32_t)m || (uint32_t)(mx - k) > (uint32_t)n) mx = OFFSET_NULL;
      mc->set(k, mx);
      ic->set(k, i1);
      dc->set(k, d1);
    }
    if (lit()) {
      const bool full = two && !affine_kernel;
      bt_affine_cells(wmm, wo1, wi1, wd1, full ? &wo2 : nullptr, full ? &wi2 : nullptr,
                      full ? &wd2 : nullptr, *mc, *ic, *dc, full ? i2c : nullptr, full ? d2c : nullptr,
                      lo, hi);
      // offload_affine / offload_affine2p (:635-705): occupancies from the
      // inputs, then every output component near full is offloaded.
      const int32_t o_i1 = occ_gap(m_open1, i1e), o_d1 = occ_gap(m_open1, d1e);
      int32_t o_m = std::max(occ_of(m_misms), std::max(o_i1, o_d1));
      int32_t o_i2 = 0, o_d2 = 0;
      if (full) {
        o_i2 = occ_gap(m_open2, i2e);
        o_d2 = occ_gap(m_open2, d2e);
        o_m = std::max(o_m, std::max(o_i2, o_d2));
      }
      ic->occ = o_i1;
      dc->occ = o_d1;
      mc->occ = o_m + 1;
      if (full) { i2c->occ = o_i2; d2c->occ = o_d2; }
      offload_component(mc, lo, hi);
      offload_component(ic, lo, hi);
      offload_component(dc, lo, hi);
      if (full) { offload_component(i2c, lo, hi); offload_component(d2c, lo, hi); }
    }
    if (two && comps.modular) {
      if (!i2c) free_wf(comps.arr[CI2][out]);
      if (!d2c) free_wf(comps.arr[CD2][out]);
    }
    comps.arr[CM][out] = mc;
    comps.arr[CI1][out] = ic;
    comps.arr[CD1][out] = dc;
    if (two) { comps.arr[CI2][out] = i2c; comps.arr[CD2][out] = d2c; }
    if (endsfree_begin_k(score, bk)) endsfree_init(*mc, bk);
    trim_ends(n, m, *mc);
    trim_ends(n, m, *ic);
    trim_ends(n, m, *dc);
    if (i2c) trim_ends(n, m, *i2c);
    if (d2c) trim_ends(n, m, *d2c);
    dominance_outputs(score);
  }

  void compute_step(int32_t score) {  // :3502-3509
    switch (pen.metric) {
      case EDIT: case INDEL: compute_edit_step(score); break;
      case LINEAR: compute_linear_step(score); break;
      default: compute_affine_step(score); break;
    }
  }

  // --- backtraces: src/backtrace.rs -----------------------------------------
  static constexpr int64_t BT_I1_OPEN = 1, BT_I1_EXT = 2, BT_I2_OPEN = 3, BT_I2_EXT = 4,
                           BT_D1_OPEN = 5, BT_D1_EXT = 6, BT_D2_OPEN = 7, BT_D2_EXT = 8, BT_M = 9;
  static inline int64_t pb(int32_t off, int64_t t) { return ((int64_t)off << 4) | t; }

  // bt_misms / bt_ins*_open / bt_del*_open / *_ext lookups, src/backtrace.rs:44-330
  int64_t bt_same(int c, int32_t score, int32_t k, int64_t type) const {
    if (score < 0) return OFFSET_NULL;
    const Wavefront* w = comps.get(c, score);
    if (!w) return OFFSET_NULL;
    if (w->init_min <= k && k <= w->init_max) return pb(w->get(k) + 1, type);
    return OFFSET_NULL;
  }
  int64_t bt_ins(int c, int32_t score, int32_t k, int64_t type) const {
    if (score < 0) return OFFSET_NULL;
    const Wavefront* w = comps.get(c, score);
    if (!w) return OFFSET_NULL;
    if (w->init_min < k && k - 1 <= w->init_max) return pb(w->get(k - 1) + 1, type);
    return OFFSET_NULL;
  }
  int64_t bt_del(int c, int32_t score, int32_t k, int64_t type) const {
    if (score < 0) return OFFSET_NULL;
    const Wavefront* w = comps.get(c, score);
    if (!w) return OFFSET_NULL;
    if (w->init_min <= k + 1 && k < w->init_max) return pb(w->get(k + 1), type);
    return OFFSET_NULL;
  }

  static void write_run(Cigar& cg, uint8_t op, int32_t n) {  // write_ops :689
    if (n <= 0) return;
    for (int32_t i = 0; i < n; ++i) cg.ops[(size_t)(cg.begin - i)] = op;
    cg.begin -= n;
  }
  static void write_matches(Cigar& cg, int32_t n) {  // :111-128
    if (n < 0) { cg.begin += -(int64_t)n; return; }
    write_run(cg, 'M', n);
  }
  static void push(Cigar& cg, uint8_t op) { cg.ops[(size_t)cg.begin] = op; cg.begin -= 1; }

  // backtrace_linear, src/backtrace.rs:132-258
  void backtrace_linear(int32_t ascore, int32_t k, int32_t offset) {
    Cigar& cg = cigar;
    cg.end = (int64_t)cg.ops.size();
    cg.begin = cg.end - 1;
    int32_t score = ascore, v = offset - k, h = offset;
    int32_t n = plen(), m = tlen();
    if (v < n) for (int32_t i = 0; i < n - v; ++i) push(cg, 'D');
    if (h < m) for (int32_t i = 0; i < m - h; ++i) push(cg, 'I');
    while (v > 0 && h > 0 && score > 0) {
      int32_t mscore = score - pen.mismatch, gscore = score - pen.o1;
      int64_t misms = pen.metric != INDEL ? bt_same(CM, mscore, k, BT_M) : (int64_t)OFFSET_NULL;
      int64_t ins = bt_ins(CM, gscore, k, BT_I1_OPEN);
      int64_t del = bt_del(CM, gscore, k, BT_D1_OPEN);
      int64_t mx = std::max(misms, std::max(ins, del));
      if (mx < 0) break;
      int32_t moff = (int32_t)(mx >> 4);
      write_matches(cg, offset - moff);
      offset = moff;
      v = offset - k; h = offset;
      if (v <= 0 || h <= 0) break;
      int64_t t = mx & 0xF;
      if (t == BT_M) { score = mscore; push(cg, 'X'); offset -= 1; }
      else if (t == BT_I1_OPEN) { score = gscore; push(cg, 'I'); k -= 1; offset -= 1; }
      else { score = gscore; push(cg, 'D'); k += 1; }
      v = offset - k; h = offset;
    }
    if (v > 0 && h > 0) {
      int32_t nm = std::min(v, h);
      write_matches(cg, nm);
      v -= nm; h -= nm;
    }
    while (v > 0) { push(cg, 'D'); --v; }
    while (h > 0) { push(cg, 'I'); --h; }
    cg.begin += 1;
    cg.score = ascore;
  }

  // backtrace_affine_c, src/backtrace.rs:492-635
  void backtrace_affine_c(int32_t ascore, int32_t k, int32_t offset, int comp_end) {
    Cigar& cg = cigar;
    bool two = pen.metric == AFFINE2P;
    cg.end = (int64_t)cg.ops.size();
    cg.begin = cg.end - 1;
    int matrix = comp_end;
    int32_t score = ascore, v = offset - k, h = offset;
    int32_t n = plen(), m = tlen();
    if (comp_end == CM) {
      for (int32_t i = 0; i < std::max(n - v, 0); ++i) push(cg, 'D');
      for (int32_t i = 0; i < std::max(m - h, 0); ++i) push(cg, 'I');
    }
    while (v > 0 && h > 0 && score > 0) {
      int32_t mis = score - pen.mismatch;
      int32_t go1 = score - pen.o1 - pen.e1, go2 = score - pen.o2 - pen.e2;
      int32_t ge1 = score - pen.e1, ge2 = score - pen.e2;
      int64_t mx;
      switch (matrix) {
        case CM: {
          int64_t misms = bt_same(CM, mis, k, BT_M);
          int64_t mi1 = std::max(bt_ins(CM, go1, k, BT_I1_OPEN), bt_ins(CI1, ge1, k, BT_I1_EXT));
          int64_t md1 = std::max(bt_del(CM, go1, k, BT_D1_OPEN), bt_del(CD1, ge1, k, BT_D1_EXT));
          if (two) {
            int64_t mi2 = std::max(bt_ins(CM, go2, k, BT_I2_OPEN), bt_ins(CI2, ge2, k, BT_I2_EXT));
            int64_t md2 = std::max(bt_del(CM, go2, k, BT_D2_OPEN), bt_del(CD2, ge2, k, BT_D2_EXT));
            mx = std::max(misms, std::max(std::max(mi1, mi2), std::max(md1, md2)));
          } else {
            mx = std::max(misms, std::max(mi1, md1));
          }
          break;
        }
        case CI1: mx = std::max(bt_ins(CM, go1, k, BT_I1_OPEN), bt_ins(CI1, ge1, k, BT_I1_EXT)); break;
        case CD1: mx = std::max(bt_del(CM, go1, k, BT_D1_OPEN), bt_del(CD1, ge1, k, BT_D1_EXT)); break;
        case CI2: mx = std::max(bt_ins(CM, go2, k, BT_I2_OPEN), bt_ins(CI2, ge2, k, BT_I2_EXT)); break;
        default: mx = std::max(bt_del(CM, go2, k, BT_D2_OPEN), bt_del(CD2, ge2, k, BT_D2_EXT)); break;
      }
      if (mx < 0) break;
      if (matrix == CM) {
        int32_t moff = (int32_t)(mx >> 4);
        write_matches(cg, offset - moff);
        offset = moff;
        v = offset - k; h = offset;
        if (v <= 0 || h <= 0) break;
      }
      int64_t t = mx & 0xF;
      switch (t) {
        case BT_M: score = mis; matrix = CM; break;
        case BT_I1_OPEN: case BT_D1_OPEN: score = go1; matrix = CM; break;
        case BT_I2_OPEN: case BT_D2_OPEN: score = go2; matrix = CM; break;
        case BT_I1_EXT: score = ge1; matrix = CI1; break;
        case BT_I2_EXT: score = ge2; matrix = CI2; break;
        case BT_D1_EXT: score = ge1; matrix = CD1; break;
        default: score = ge2; matrix = CD2; break;
      }
      if (t == BT_M) { push(cg, 'X'); offset -= 1; }
      else if (t == BT_I1_OPEN || t == BT_I1_EXT || t == BT_I2_OPEN || t == BT_I2_EXT) {
        push(cg, 'I'); k -= 1; offset -= 1;
      } else { push(cg, 'D'); k += 1; }
      v = offset - k; h = offset;
    }
    if (matrix == CM) {
      if (v > 0 && h > 0) {
        int32_t nm = std::min(v, h);
        write_matches(cg, nm);
        v -= nm; h -= nm;
      }
      for (int32_t i = 0; i < v; ++i) push(cg, 'D');
      for (int32_t i = 0; i < h; ++i) push(cg, 'I');
    }
    cg.begin += 1;
    cg.score = ascore;
  }

  // st_m_offset, src/backtrace.rs:645-663
  bool st_m_offset(int32_t score, int32_t k, int32_t& out) const {
    if (score < 0 || !comps.has_slot(score)) return false;
    const Wavefront* w = comps.get(CM, score);
    if (!w) return false;
    if (k < w->init_min || w->init_max < k) return false;
    int32_t o = w->get(k);
    if (o == OFFSET_NULL) return false;
    out = o;
    return true;
  }
  // st_backward_matches, src/backtrace.rs:668-686
  int32_t st_backward_matches(int32_t v, int32_t h) const {
    int32_t mx = std::min(v, h), n = 0;
    const uint8_t* P = seq.P();
    const uint8_t* T = seq.T();
    while (n < mx && P[v - 1 - n] == T[h - 1 - n]) ++n;
    return n;
  }
  // st_gap, src/backtrace.rs:707-737
  bool st_gap(int32_t gscore, int32_t l, int32_t off_orig, int32_t& k, int32_t& offset) {
    int32_t mo;
    if (st_m_offset(gscore, k - l, mo) && mo + l >= off_orig && mo + l <= offset) {
      write_run(cigar, 'M', offset - (mo + l));
      write_run(cigar, 'I', l);
      k -= l;
      offset = mo;
      return true;
    }
    if (st_m_offset(gscore, k + l, mo) && mo >= off_orig && mo <= offset) {
      write_run(cigar, 'M', offset - mo);
      write_run(cigar, 'D', l);
      k += l;
      offset = mo;
      return true;
    }
    return false;
  }
  // backtrace_affine_singletrack, src/backtrace.rs:751-858
  void backtrace_singletrack(int32_t pbf, int32_t tbf, int32_t ascore, int32_t k, int32_t offset) {
    (void)pbf; (void)tbf;
    Cigar& cg = cigar;
    bool two = pen.metric == AFFINE2P;
    cg.end = (int64_t)cg.ops.size();
    cg.begin = cg.end - 1;
    int32_t score = ascore, off_orig = offset;
    write_run(cg, 'D', plen() - (offset - k));
    write_run(cg, 'I', tlen() - offset);
    bool in_m = true;
    int32_t l = 0;
    while (score != 0) {
      if (in_m) {
        int32_t nm = st_backward_matches(offset - k, offset);
        off_orig = offset - nm;
        int32_t mis = score - pen.mismatch, mo;
        if (st_m_offset(mis, k, mo) && mo == off_orig - 1) {
          write_run(cg, 'M', nm);
          write_run(cg, 'X', 1);
          offset = off_orig - 1;
          score = mis;
        } else {
          in_m = false;
          l = 0;
        }
      } else {
        ++l;
        int32_t ind1 = score - pen.o1 - l * pen.e1;
        int32_t ind2 = two ? score - pen.o2 - l * pen.e2 : -1;
        if (st_gap(ind1, l, off_orig, k, offset)) { score = ind1; in_m = true; }
        else if (st_gap(ind2, l, off_orig, k, offset)) { score = ind2; in_m = true; }
        else if (ind1 < 0 && ind2 < 0) {
          in_m = (off_orig - k) == 0 || off_orig == 0;
          break;
        }
      }
    }
    int32_t v = offset - k, h = offset;
    int32_t nm = std::min(v, h);
    v -= nm; h -= nm;
    write_run(cg, 'M', nm);
    write_run(cg, 'D', v);
    write_run(cg, 'I', h);
    cg.begin += 1;
    cg.score = ascore;
  }

  bool singletrack() const {  // src/aligner.rs:1366-1373
    return !comps.modular && (pen.metric == AFFINE || pen.metric == AFFINE2P);
  }
  void backtrace_components(int32_t score, int32_t k, int32_t off, int /*cb*/, int ce) {  // :1489
    if (pen.metric == AFFINE || pen.metric == AFFINE2P) backtrace_affine_c(score, k, off, ce);
    else backtrace_linear(score, k, off);
  }
  void backtrace_from(int32_t score, int32_t k, int32_t off) {  // :1414-1436
    if (piggyback) {
      backtrace_piggyback(score, k, off);
    } else if (singletrack()) {
      int32_t pbf = span == SPAN_ENDSFREE ? p0 : 0, tbf = span == SPAN_ENDSFREE ? t0 : 0;
      backtrace_singletrack(pbf, tbf, score, k, off);
    } else {
      backtrace_components(score, k, off, CM, CM);
    }
  }
  void backtrace_zdrop_end(int32_t score) {  // :1393-1411
    // C: med/low read the end cell at the current score (where it may be
    // dead).  Corrected: every mode backtraces the best cell at the score it
    // was found at (med/low from the backtrace kept then; every score's
    // cells are kept here, so that is the cell's own chain).
    if (compat == 1 && lit()) {
      backtrace_piggyback_bt(zdrop_bt_pc, zdrop_bt_pv, end_pos.score, end_pos.k, end_pos.offset);
      return;
    }
    int32_t from = compat == 1 ? end_pos.score
                   : (!piggyback && end_pos.score >= 0) ? end_pos.score : score;
    backtrace_from(from, end_pos.k, end_pos.offset);
  }

  // --- med/low: the piggyback backtrace --------------------------------------
  // Offset of (comp, score, k) as the compute kernels read it (absent and
  // null wavefronts read as NULL).
  int32_t pv(int comp, int32_t s, int32_t k) const {
    if (s < 0) return OFFSET_NULL;
    const Wavefront* w = comps.get(comp, s);
    if (is_null_wf(w)) return OFFSET_NULL;
    return w->get(k);
  }
  struct Step {
    uint8_t op;
    int comp;
    int32_t s, k;
  };
  // The predecessor a piggyback kernel copied cell (comp, s, k)'s backtrace
  // from, and the operation it pushed (src/compute/piggyback.rs:172-528):
  // edit/linear take misms over del over ins (later checks win ties), indel
  // del over ins; a gap cell takes its extension over the M opening on a tie
  // (`gap`, :146-170); affine M takes misms, else D2, D1, I2, I1 in that
  // order, pushing an X on top of the gap's chain (the gap close, dropped
  // when unpacking).
  Step piggyback_pred(int comp, int32_t s, int32_t k) const {
    const int32_t x = pen.mismatch;
    switch (pen.metric) {
      case EDIT: case INDEL: case LINEAR: {
        const int32_t gs = pen.metric == LINEAR ? s - pen.o1 : s - 1;
        const int32_t ms = pen.metric == LINEAR ? s - x : s - 1;
        const int32_t ins = wrap_add(pv(CM, gs, k - 1), 1), del = pv(CM, gs, k + 1);
        if (pen.metric == INDEL) {
          const int32_t mx = std::max(del, ins);
          return mx == del ? Step{'D', CM, gs, k + 1} : Step{'I', CM, gs, k - 1};
        }
        const int32_t misms = wrap_add(pv(CM, ms, k), 1);
        const int32_t mx = std::max(del, std::max(ins, misms));
        if (mx == misms) return Step{'X', CM, ms, k};
        return mx == del ? Step{'D', CM, gs, k + 1} : Step{'I', CM, gs, k - 1};
      }
      default: {
        const bool two = pen.metric == AFFINE2P;
        if (comp == CI1 || comp == CD1 || comp == CI2 || comp == CD2) {
          const bool ins = comp == CI1 || comp == CI2;
          const bool p2 = comp == CI2 || comp == CD2;
          const int32_t o = p2 ? pen.o2 : pen.o1, e = p2 ? pen.e2 : pen.e1;
          const int32_t kk = ins ? k - 1 : k + 1;
          const int32_t open = pv(CM, s - o - e, kk), ext = pv(comp, s - e, kk);
          const uint8_t op = ins ? 'I' : 'D';
          return ext >= open ? Step{op, comp, s - e, kk} : Step{op, CM, s - o - e, kk};
        }
        const int32_t i1 = pv(CI1, s, k), d1 = pv(CD1, s, k);
        const int32_t i2 = two ? pv(CI2, s, k) : OFFSET_NULL, d2 = two ? pv(CD2, s, k) : OFFSET_NULL;
        const int32_t misms = wrap_add(pv(CM, s - x, k), 1);
        int32_t mx = std::max(d1, std::max(misms, i1));
        if (two) mx = std::max(std::max(std::max(i1, i2), std::max(d1, d2)), misms);
        if (mx == misms) return Step{'X', CM, s - x, k};
        if (two && mx == d2) return Step{'X', CD2, s, k};
        if (mx == d1) return Step{'X', CD1, s, k};
        if (two && mx == i2) return Step{'X', CI2, s, k};
        return Step{'X', CI1, s, k};
      }
    }
  }

  // backtrace_piggyback, src/aligner.rs:1443-1459: the end cell's chain.
  void backtrace_piggyback(int32_t score, int32_t k, int32_t offset) {
    if (!bt_literal) { backtrace_piggyback_rederived(score, k, offset); return; }
    const Wavefront* m = comps.get(CM, score);
    if (!m || !m->allocated(k)) { cigar.begin = 0; cigar.end = 0; return; }
    uint32_t c, v;
    m->bt_or_zero(k, c, v);
    backtrace_piggyback_bt(c, v, score, k, offset);
  }
  // backtrace_piggyback_bt, :1463-1486: the blocks back to the initial one
  // (traceback_from), unpacked from the initial position.
  void backtrace_piggyback_bt(uint32_t pc, uint32_t pv, int32_t score, int32_t k, int32_t offset) {
    const uint32_t init = bt.traceback_from(pc, pv);
    const auto ip = bt.init_pos[init];
    unpack_packed(bt.packed, ip.first, ip.second, offset - k, offset);
    cigar.score = score;
  }
  // unpack_piggyback, :232-311, on packed blocks (end first): begin-free I
  // then D, each block's operations from its first, matches re-extended
  // before each (only in M when affine, where an X after I/D is the gap
  // close and is dropped), matches to the end cell (a negative count moves
  // back), then I and D to the sequence ends.
  void unpack_packed(const std::vector<uint32_t>& packed, int32_t v, int32_t h, int32_t end_v,
                     int32_t end_h) {
    const int32_t n = plen(), m = tlen();
    const bool affine = pen.metric == AFFINE || pen.metric == AFFINE2P;
    int64_t p = 0;
    auto put = [&](uint8_t op) { cigar.ops[(size_t)p++] = op; };
    for (int32_t i = 0; i < h; ++i) put('I');
    for (int32_t i = 0; i < v; ++i) put('D');
    bool in_m = true;
    for (size_t b = packed.size(); b-- > 0;) {
      uint32_t pcig = packed[b];
      int32_t length = PCIGAR_MAX_LENGTH;
      if (pcig < PCIGAR_FULL_MASK) {
        const int32_t fr = pcigar_free_slots(pcig);
        length -= fr;
        pcig = fr >= 16 ? 0u : pcig << (2 * fr);
      }
      for (int32_t j = 0; j < length; ++j) {
        if (in_m || !affine) {
          while (v < n && h < m && seq.cmp(v, h)) { put('M'); ++v; ++h; }
        }
        const uint32_t op = pcig >> 30;
        pcig <<= 2;
        uint8_t ch;
        int32_t dv, dh;
        bool mm;
        if (op == PCIGAR_DELETION) { ch = 'D'; dv = 1; dh = 0; mm = false; }
        else if (op == PCIGAR_MISMATCH) { ch = 'X'; dv = 1; dh = 1; mm = true; }
        else if (op == PCIGAR_INSERTION) { ch = 'I'; dv = 0; dh = 1; mm = false; }
        else { ch = '?'; dv = 0; dh = 0; mm = true; }
        if (affine && !in_m && ch == 'X') { in_m = true; continue; }
        put(ch);
        v += dv;
        h += dh;
        in_m = mm;
      }
    }
    const int32_t nm = std::min(end_v - v, end_h - h);
    for (int32_t i = 0; i < nm; ++i) put('M');
    v += nm;
    h += nm;
    while (h < m) { put('I'); ++h; }
    while (v < n) { put('D'); ++v; }
    cigar.begin = 0;
    cigar.end = p;
  }

  // The same chain re-made from the kept offsets: each step applies the
  // kernels' tie order to the stored predecessors (piggyback_pred).
  void backtrace_piggyback_rederived(int32_t score, int32_t k, int32_t offset) {
    const Wavefront* m = comps.get(CM, score);
    if (!m || !m->allocated(k)) { cigar.begin = 0; cigar.end = 0; return; }
    std::vector<uint8_t> back;
    int32_t bv = 0, bh = 0;  // the chain's begin; (0, 0) for an unwritten cell
    int comp = CM;
    int32_t s = score, kk = k;
    const Wavefront* w = m;
    // A cell outside the written range (or a dead cell, whose backtrace the
    // kernels never build from a live predecessor) reads as the zero
    // backtrace: no operations, from the first initial block (0, 0).
    while (w && w->written(kk) && w->get(kk) >= 0) {
      if (comp == CM && (s == 0 || w->is_seed(kk))) {
        // The seed's position when it was placed (before any extension):
        // (0, k) on a text diagonal, (-k, 0) on a pattern one, (0, 0) at k 0.
        bv = kk < 0 ? -kk : 0;
        bh = kk > 0 ? kk : 0;
        break;
      }
      const Step st = piggyback_pred(comp, s, kk);
      back.push_back(st.op);
      comp = st.comp; s = st.s; kk = st.k;
      w = s >= 0 ? comps.get(comp, s) : nullptr;
      if (is_null_wf(w)) break;
    }
    std::reverse(back.begin(), back.end());
    unpack_piggyback(back, bv, bh, offset - k, offset);
    cigar.score = score;
  }

  // unpack_piggyback, src/aligner.rs:232-311: begin-free I/D, then the
  // operations, re-extending matches before each one (only in M when
  // affine, where an X after I/D is the gap close and is dropped), then
  // matches to the end cell and I/D to the sequence ends.
  void unpack_piggyback(const std::vector<uint8_t>& ops, int32_t v, int32_t h, int32_t end_v,
                        int32_t end_h) {
    const int32_t n = plen(), m = tlen();
    const bool affine = pen.metric == AFFINE || pen.metric == AFFINE2P;
    int64_t p = 0;
    auto put = [&](uint8_t op) { cigar.ops[(size_t)p++] = op; };
    for (int32_t i = 0; i < h; ++i) put('I');
    for (int32_t i = 0; i < v; ++i) put('D');
    bool in_m = true;
    for (uint8_t op : ops) {
      if (in_m || !affine) {
        while (v < n && h < m && seq.cmp(v, h)) { put('M'); ++v; ++h; }
      }
      if (affine && !in_m && op == 'X') { in_m = true; continue; }
      put(op);
      if (op == 'D') { ++v; in_m = false; }
      else if (op == 'I') { ++h; in_m = false; }
      else { ++v; ++h; in_m = true; }
    }
    const int32_t nm = std::min(end_v - v, end_h - h);
    for (int32_t i = 0; i < nm; ++i) put('M');
    v += nm;
    h += nm;
    while (h < m) { put('I'); ++h; }
    while (v < n) { put('D'); ++v; }
    cigar.begin = 0;
    cigar.end = p;
  }

  // cigar_wfa_score, src/aligner.rs:2700-2719
  int32_t cigar_wfa_score(const Cigar& cg, int32_t n, int32_t m) const {
    int32_t classic;
    switch (pen.metric) {
      case INDEL: case EDIT: return cg.score_edit();
      case LINEAR: classic = cg.score_gap_linear(pen.orig); break;
      case AFFINE: classic = cg.score_gap_affine(pen.orig); break;
      default: classic = cg.score_gap_affine2p(pen.orig); break;
    }
    if (pen.match_ < 0) return -pen.match_ * (n + m) - 2 * classic;
    return -classic;
  }
  int32_t cigar_skip_gap(uint8_t op, int32_t maxlen) {  // :1580-1592
    int32_t len = 0;
    while (len < maxlen && cigar.begin < cigar.end && cigar.ops[(size_t)cigar.begin] == op) {
      ++cigar.begin;
      ++len;
    }
    return len;
  }
  // maxtrim_cigar, src/aligner.rs:1545-1577
  bool maxtrim_cigar() {
    if (pen.metric == EDIT || pen.metric == INDEL) return false;
    int32_t bv = 0, bh = 0;
    if (span == SPAN_ENDSFREE) {
      bh = cigar_skip_gap('I', t0);
      if (bh == 0) bv = cigar_skip_gap('D', p0);
    }
    if (cigar.begin >= cigar.end) { cigar.clear(); return true; }
    bool trimmed;
    if (pen.metric == LINEAR) trimmed = cigar.maxtrim_simple(pen.orig, false);
    else if (pen.metric == AFFINE) trimmed = cigar.maxtrim_simple(pen.orig, true);
    else trimmed = cigar.maxtrim_gap_affine2p(pen.orig);
    if (cigar.score != INT32_MIN) {
      cigar.score = cigar_wfa_score(cigar, cigar.end_v, cigar.end_h);
      cigar.begin -= bv + bh;
      cigar.end_v += bv;
      cigar.end_h += bh;
    }
    return trimmed;
  }
  // rescore_heuristic_cigar, src/aligner.rs:1605-1640
  int32_t rescore_heuristic_cigar(int32_t score) {
    if (heur.kind == H_NONE || !(pen.metric == AFFINE || pen.metric == AFFINE2P)) return score;
    int64_t b = cigar.begin, e = cigar.end;
    if (span == SPAN_ENDSFREE) {
      int32_t trailing = (plen() - cigar.end_v) + (tlen() - cigar.end_h);
      // end.saturating_sub(trailing as usize): a negative count wraps to a
      // huge usize, so the view becomes empty.
      cigar.end = trailing < 0 ? 0 : std::max<int64_t>(0, e - trailing);
      uint8_t op = b < (int64_t)cigar.ops.size() ? cigar.ops[(size_t)b] : 0;
      int32_t fr = op == 'I' ? t0 : op == 'D' ? p0 : 0;
      cigar_skip_gap(op, fr);
    }
    int64_t vb = cigar.begin, ve = std::max(cigar.end, vb);
    int32_t rescored = 0;
    if (ve > vb) {
      int32_t v = 0, h = 0;
      for (int64_t i = vb; i < ve; ++i) { v += cigar.ops[(size_t)i] != 'I'; h += cigar.ops[(size_t)i] != 'D'; }
      Cigar view = cigar;
      view.begin = vb;
      view.end = ve;
      rescored = cigar_wfa_score(view, v, h);
    }
    cigar.begin = b;
    cigar.end = e;
    cigar.score = rescored;
    return rescored;
  }

  // --- public aligners ------------------------------------------------------
  // align_end2end_span, src/aligner.rs:638-698
  int32_t align_end2end_span() {
    init_alignment();
    int32_t score = 0;
    for (;;) {
      if (extend_end2end(score)) break;
      ++score;
      if (!comps.make_slot(score)) { status = MAX_STEPS; break; }
      compute_step(score);
      if (score >= max_steps) { status = MAX_STEPS; break; }
    }
    int32_t result = score;
    if (status == END_REACHED) {
      if (scope == SCOPE_ALIGNMENT) {
        backtrace_from(score, end_pos.k, end_pos.offset);
        cigar.end_v = end_pos.offset - end_pos.k;
        cigar.end_h = end_pos.offset;
        result = rescore_heuristic_cigar(score);
      }
      status = COMPLETED;
    } else if (status == END_UNREACHABLE && end_pos.offset != OFFSET_NULL) {
      if (scope == SCOPE_ALIGNMENT) {
        backtrace_zdrop_end(score);
        maxtrim_cigar();
      }
      status = PARTIAL;
    }
    if (scope == SCOPE_ALIGNMENT) ctr.ops = cigar.end - cigar.begin;
    return result;
  }
  int32_t align_end2end_inner() {  // :627-635
    int saved = span;
    span = SPAN_END2END;
    int32_t r = align_end2end_span();
    span = saved;
    return r;
  }
  int32_t align_end2end(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {  // :620
    seq.init_ascii(p, n, t, m, false);
    return align_end2end_inner();
  }
  int32_t align_packed2bits(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {  // :2755
    std::vector<uint8_t> pa = decode_packed2bits(p, n), ta = decode_packed2bits(t, m);
    seq.init_ascii(pa.data(), n, ta.data(), m, false);
    return align_end2end_inner();
  }

  // align_endsfree, src/aligner.rs:707-831 (C compatibility)
  int32_t align_endsfree(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
    seq.init_ascii(p, n, t, m, false);
    if (extension) { p0 = 0; pf = n; t0 = 0; tf = m; }
    init_alignment();
    int32_t score = 0;
    for (;;) {
      if (extend_endsfree(score)) break;
      ++score;
      if (!comps.make_slot(score)) { status = MAX_STEPS; break; }
      compute_step(score);
      if (score >= max_steps) { status = MAX_STEPS; break; }
    }
    int32_t result = score;
    if (status == END_REACHED || status == END_UNREACHABLE) {
      bool unreachable = status == END_UNREACHABLE;
      // Corrected mode: the candidate's cell can be from an earlier score,
      // and its total is the alignment's score (:772-777).
      const bool cand = best.has && !unreachable;
      if (cand) result = best.total;
      if (scope == SCOPE_ALIGNMENT && (status == END_REACHED || end_pos.offset != OFFSET_NULL)) {
        if (cand) {
          if (lit()) backtrace_piggyback_bt(best.bt_pc, best.bt_pv, best.pos.score, best.pos.k, best.pos.offset);
          else backtrace_from(best.pos.score, best.pos.k, best.pos.offset);
          cigar.score = best.total;
        } else if (unreachable) {
          backtrace_zdrop_end(score);
        } else {
          backtrace_from(score, end_pos.k, end_pos.offset);
        }
        if (extension || unreachable) {
          bool trimmed = maxtrim_cigar();
          status = (trimmed || unreachable) ? PARTIAL : COMPLETED;
        } else {
          cigar.end_v = end_pos.offset - end_pos.k;
          cigar.end_h = end_pos.offset;
          if (!cand) result = rescore_heuristic_cigar(score);
          status = COMPLETED;
        }
      } else {
        status = unreachable ? PARTIAL : COMPLETED;
      }
    }
    if (scope == SCOPE_ALIGNMENT) ctr.ops = cigar.end - cigar.begin;
    return result;
  }

  // --- BiWFA: src/aligner.rs:2563-3202, 3244-3302, 3516-3554 ----------------
  static std::unique_ptr<Aligner> new_biwfa_sub(const Penalties& p) {  // :2768
    std::unique_ptr<Aligner> a(new Aligner(p));
    a->comps.create(10, 10, p, true);
    a->scope = SCOPE_SCORE;
    return a;
  }
  void take_biwfa_subs() {  // :2721-2741
    if (!bi_fwd) {
      bi_fwd = new_biwfa_sub(pen);
      bi_rev = new_biwfa_sub(pen);
      bi_base.reset(new Aligner(pen));
      bi_base->scope = SCOPE_ALIGNMENT;
    }
    bi_base->compat = compat;
  }
  // check_component_termination, :3268-3302
  bool check_component_termination(int32_t score, int comp) {
    int32_t kend = tlen() - plen();
    const Wavefront* w = comps.get(comp, score);
    if (!w) return false;
    if (kend >= w->lo && kend <= w->hi && w->get(kend) >= tlen()) {
      end_pos = Pos{score, kend, tlen()};
      status = END_REACHED;
      return true;
    }
    return false;
  }
  // extend_biwfa_step, :3516-3554
  bool extend_biwfa_step(int32_t score, int comp_end, bool max, int32_t& max_ak) {
    max_ak = 0;
    Wavefront* m = comps.get(CM, score);
    if (!m) {
      if (num_null_steps > (int32_t)comps.scope) { status = END_UNREACHABLE; return true; }
      return false;
    }
    int32_t ak = 0;
    if (max) ak = extend_end2end_max_wf(*m);
    else extend_end2end_wf(*m);
    if (check_component_termination(score, comp_end)) return true;
    if (heur.kind != H_NONE && apply_heuristic_cutoff(score, m)) {
      status = END_UNREACHABLE;
      return true;
    }
    max_ak = ak;
    return false;
  }

  // bialign_find_breakpoint, :2958-3124
  static BiStatus find_breakpoint(const Penalties& pen, int32_t max_steps, Aligner& fwd,
                                  Aligner& rev, const uint8_t* P, int32_t n, const uint8_t* T,
                                  int32_t m, int cb, int ce, Breakpoint& bp) {
    fwd.seq.init_ascii(P, n, T, m, false);
    fwd.init_alignment_component(cb);
    rev.seq.init_ascii(P, n, T, m, true);
    rev.init_alignment_component(ce);
    int fwd_end = ce, rev_end = cb;
    auto quit = [](const Aligner& a) {
      BiStatus s;
      if (a.status == END_REACHED) { s.kind = BI_END_REACHED; s.score = a.end_pos.score; }
      else s.kind = BI_UNREACHABLE;
      return s;
    };
    bool has_affine = pen.metric == AFFINE || pen.metric == AFFINE2P;
    bool has_2p = pen.metric == AFFINE2P;
    int32_t gap_opening = pen.metric == AFFINE ? pen.o1 : pen.metric == AFFINE2P ? std::max(pen.o1, pen.o2) : 0;
    int32_t max_ad = n + m - 1;
    int32_t sf = 0, sr = 0;
    bool last_fwd = false;
    int32_t fak, rak, ak;
    if (fwd.extend_biwfa_step(0, fwd_end, true, fak)) return quit(fwd);
    if (rev.extend_biwfa_step(0, rev_end, true, rak)) return quit(rev);
    while (fak + rak < max_ad) {
      ++sf;
      fwd.compute_step(sf);
      bool done = fwd.extend_biwfa_step(sf, fwd_end, true, ak);
      fak = std::max(fak, ak);
      last_fwd = true;
      if (done) return quit(fwd);
      if (fak + rak >= max_ad) break;
      ++sr;
      rev.compute_step(sr);
      done = rev.extend_biwfa_step(sr, rev_end, true, ak);
      rak = std::max(rak, ak);
      last_fwd = false;
      if (done) return quit(rev);
      if (sf + sr >= max_steps) { BiStatus s; s.kind = BI_MAXSTEPS; return s; }
    }
    int32_t scope = (int32_t)fwd.comps.scope;
    for (;;) {
      if (last_fwd) {
        int32_t min_sr = sr > scope - 1 ? sr - (scope - 1) : 0;
        if (sf + min_sr - gap_opening >= bp.score) break;
        bialign_overlap(fwd.comps, rev.comps, sf, sr, n, m, pen.o1, pen.o2, has_affine, has_2p, true, bp);
        ++sr;
        rev.compute_step(sr);
        if (rev.extend_biwfa_step(sr, rev_end, false, ak)) return quit(rev);
      }
      int32_t min_sf = sf > scope - 1 ? sf - (scope - 1) : 0;
      if (min_sf + sr - gap_opening >= bp.score) break;
      bialign_overlap(rev.comps, fwd.comps, sr, sf, n, m, pen.o1, pen.o2, has_affine, has_2p, false, bp);
      ++sf;
      fwd.compute_step(sf);
      if (fwd.extend_biwfa_step(sf, fwd_end, false, ak)) return quit(fwd);
      if (sf + sr >= max_steps) { BiStatus s; s.kind = BI_MAXSTEPS; return s; }
      last_fwd = true;
    }
    return BiStatus();
  }

  // bialign_base, :3127-3202
  static BiStatus bialign_base(Cigar& out, const Heuristic& h, Aligner& base, const uint8_t* P,
                               const uint8_t* T, int32_t pb_, int32_t pe, int32_t tb, int32_t te,
                               int cb, int ce, int32_t& result) {
    base.heur = h.banded() ? h.with_band(h.p0 - (tb - pb_), h.p1 - (tb - pb_)) : h;
    base.seq.init_ascii(P + pb_, pe - pb_, T + tb, te - tb, false);
    base.init_alignment_component(cb);
    int32_t score = 0, ak;
    for (;;) {
      if (base.extend_biwfa_step(score, ce, false, ak)) break;
      ++score;
      if (!base.comps.has_slot(score)) { base.status = MAX_STEPS; break; }
      base.compute_step(score);
      if (score >= base.max_steps) { base.status = MAX_STEPS; break; }
    }
    Pos pos = base.end_pos;
    BiStatus st;
    if (base.status == END_REACHED) {
      base.backtrace_components(score, pos.k, pos.offset, cb, ce);
      result = score;
    } else if (base.status == END_UNREACHABLE && pos.offset != OFFSET_NULL) {
      // C: from component_end at the best cell's score; Corrected: from M
      // (the best cell is an M cell), :3181-3192.
      if (base.compat == 1) {
        base.backtrace_components(pos.score, pos.k, pos.offset, cb, CM);
      } else {
        int32_t from = pos.score >= 0 ? pos.score : score;
        base.backtrace_components(from, pos.k, pos.offset, cb, ce);
      }
      base.maxtrim_cigar();
      st.kind = BI_UNATTAINABLE;
    } else {
      base.cigar.clear();
      st.kind = BI_UNATTAINABLE;
    }
    out.append_forward(base.cigar);
    return st;
  }

  // bialign_recursive, :2809-2950
  static BiStatus bialign_recursive(Cigar& cg, const Penalties& pen, const Heuristic& h,
                                    int32_t max_steps, Aligner& fwd, Aligner& rev, Aligner& base,
                                    const uint8_t* P, const uint8_t* T, int32_t pb_, int32_t pe,
                                    int32_t tb, int32_t te, int cb, int ce,
                                    int32_t score_remaining, int32_t& result) {
    int32_t n = pe - pb_, m = te - tb;
    if (m == 0) { if (n > 0) cg.append_deletion(n); result = 0; return BiStatus(); }
    if (n == 0) { if (m > 0) cg.append_insertion(m); result = 0; return BiStatus(); }
    if (score_remaining <= BIALIGN_FALLBACK_MIN_SCORE)
      return bialign_base(cg, h, base, P, T, pb_, pe, tb, te, cb, ce, result);
    fwd.heur = h;
    rev.heur = h;
    if (h.banded()) {
      int32_t shift = tb - pb_;
      int32_t fmin = h.p0 - shift, fmax = h.p1 - shift, diag = m - n;
      fwd.heur = h.with_band(fmin, fmax);
      rev.heur = h.with_band(diag - fmax, diag - fmin);
    }
    Breakpoint bp;
    BiStatus st = find_breakpoint(pen, max_steps, fwd, rev, P + pb_, n, T + tb, m, cb, ce, bp);
    if (st.kind == BI_END_REACHED) {
      if (st.score <= BIALIGN_RECOVERY_MIN_SCORE)
        return bialign_base(cg, h, base, P, T, pb_, pe, tb, te, cb, ce, result);
      BiStatus u;
      u.kind = BI_UNREACHABLE;
      return u;
    }
    if (st.kind != BI_OK) return st;
    int32_t bph = bp.offset_forward, bpv = bp.offset_forward - bp.k_forward;
    int32_t r1, r2;
    st = bialign_recursive(cg, pen, h, max_steps, fwd, rev, base, P, T, pb_, pb_ + bpv, tb,
                           tb + bph, cb, bp.component, bp.score_forward, r1);
    if (st.kind != BI_OK) return st;
    st = bialign_recursive(cg, pen, h, max_steps, fwd, rev, base, P, T, pb_ + bpv, pe, tb + bph,
                           te, bp.component, ce, bp.score_reverse, r2);
    if (st.kind != BI_OK) return st;
    result = bp.score;
    return BiStatus();
  }

  // align_biwfa, :2563-2644
  int32_t align_biwfa(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
    seq.init_ascii(p, n, t, m, false);
    scope = SCOPE_ALIGNMENT;
    cigar.resize((size_t)(2 * (n + m)) + 1);
    status = OK;
    take_biwfa_subs();
    int32_t result = 0;
    BiStatus st = bialign_recursive(cigar, pen, heur, max_steps, *bi_fwd, *bi_rev, *bi_base, p, t, 0, n,
                                    0, m, CM, CM, std::max(n, m) <= BIALIGN_FALLBACK_MIN_LENGTH ? 0 : INT32_MAX,
                                    result);
    int32_t score;
    if (st.kind == BI_OK) {
      bool h = heur.kind != H_NONE && cigar.begin < cigar.end;
      score = (n == 0 || m == 0 || h) ? cigar_wfa_score(cigar, n, m) : result;
      cigar.score = score;
      cigar.end_v = n;
      cigar.end_h = m;
      status = COMPLETED;
    } else {
      status = st.kind == BI_MAXSTEPS ? MAX_STEPS : END_UNREACHABLE;
      score = 0;
    }
    ctr.ops = cigar.end - cigar.begin;
    return score;
  }
  // align_biwfa_score, :2650-2698
  int32_t align_biwfa_score(const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
    seq.init_ascii(p, n, t, m, false);
    cigar.clear();
    take_biwfa_subs();
    bi_fwd->heur = heur;
    bi_rev->heur = heur;
    if (heur.banded()) {
      int32_t diag = m - n;
      bi_rev->heur = heur.with_band(diag - heur.p1, diag - heur.p0);
    }
    Breakpoint bp;
    BiStatus st = find_breakpoint(pen, max_steps, *bi_fwd, *bi_rev, p, n, t, m, CM, CM, bp);
    int32_t score = st.kind == BI_OK ? bp.score : st.kind == BI_END_REACHED ? st.score : 0;
    status = (st.kind == BI_OK || st.kind == BI_END_REACHED) ? COMPLETED
             : st.kind == BI_MAXSTEPS ? MAX_STEPS : END_UNREACHABLE;
    return score;
  }
};

}  // namespace wfo

using namespace wfo;

// ---------------------------------------------------------------------------
// C interface
// ---------------------------------------------------------------------------
extern "C" {

void* wfo_create(int metric, const int32_t* pen) {
  Penalties p;
  int32_t zero[6] = {0, 0, 0, 0, 0, 0};
  if (!make_penalties(metric, pen ? pen : zero, p)) return nullptr;
  return new Aligner(p);
}
void wfo_destroy(void* h) { delete static_cast<Aligner*>(h); }
void wfo_set_alignment_scope(void* h, int a) { static_cast<Aligner*>(h)->scope = a ? SCOPE_ALIGNMENT : SCOPE_SCORE; }
void wfo_set_memory_mode(void* h, int mode) { static_cast<Aligner*>(h)->memory_mode = mode; }
void wfo_set_compat(void* h, int compat) { static_cast<Aligner*>(h)->compat = compat; }
void wfo_set_piggyback_literal(void* h, int on) { static_cast<Aligner*>(h)->bt_literal = on != 0; }
void wfo_set_heuristic(void* h, int kind, int32_t p0, int32_t p1, int32_t p2) {
  Heuristic& hs = static_cast<Aligner*>(h)->heur;
  hs.kind = kind; hs.p0 = p0; hs.p1 = p1; hs.p2 = p2;
}
void wfo_set_max_alignment_steps(void* h, int32_t s) { static_cast<Aligner*>(h)->max_steps = s; }
void wfo_set_alignment_free_ends(void* h, int32_t p0, int32_t pf, int32_t t0, int32_t tf) {
  Aligner* a = static_cast<Aligner*>(h);  // :563-576
  a->span = SPAN_ENDSFREE; a->extension = false;
  a->p0 = p0; a->pf = pf; a->t0 = t0; a->tf = tf;
}
void wfo_set_alignment_extension(void* h) {  // :582-585
  Aligner* a = static_cast<Aligner*>(h);
  a->span = SPAN_ENDSFREE; a->extension = true;
}
void wfo_set_alignment_end_to_end(void* h) {  // :595-603
  Aligner* a = static_cast<Aligner*>(h);
  a->span = SPAN_END2END; a->extension = false; a->p0 = a->pf = a->t0 = a->tf = 0;
}
int32_t wfo_align_end2end(void* h, const char* p, int32_t n, const char* t, int32_t m) {
  return static_cast<Aligner*>(h)->align_end2end((const uint8_t*)p, n, (const uint8_t*)t, m);
}
int32_t wfo_align_endsfree(void* h, const char* p, int32_t n, const char* t, int32_t m) {
  return static_cast<Aligner*>(h)->align_endsfree((const uint8_t*)p, n, (const uint8_t*)t, m);
}
int32_t wfo_align_biwfa(void* h, const char* p, int32_t n, const char* t, int32_t m) {
  return static_cast<Aligner*>(h)->align_biwfa((const uint8_t*)p, n, (const uint8_t*)t, m);
}
int32_t wfo_align_biwfa_score(void* h, const char* p, int32_t n, const char* t, int32_t m) {
  return static_cast<Aligner*>(h)->align_biwfa_score((const uint8_t*)p, n, (const uint8_t*)t, m);
}
int32_t wfo_align_packed2bits(void* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m) {
  return static_cast<Aligner*>(h)->align_packed2bits(p, n, t, m);
}
int wfo_status(void* h) { return static_cast<Aligner*>(h)->status; }
int32_t wfo_cigar(void* h, char* ops, int32_t cap, int32_t* score, int32_t* ev, int32_t* eh) {
  Aligner* a = static_cast<Aligner*>(h);
  const Cigar& c = a->cigar;
  int32_t len = c.empty() ? 0 : (int32_t)(c.end - c.begin);
  for (int32_t i = 0; i < len && i < cap; ++i) ops[i] = (char)c.ops[(size_t)(c.begin + i)];
  if (score) *score = c.score;
  if (ev) *ev = c.end_v;
  if (eh) *eh = c.end_h;
  return len;
}
void wfo_end_pos(void* h, int32_t* s, int32_t* k, int32_t* o) {
  Aligner* a = static_cast<Aligner*>(h);
  if (s) *s = a->end_pos.score;
  if (k) *k = a->end_pos.k;
  if (o) *o = a->end_pos.offset;
}
void wfo_counters(void* h, int64_t* cells, int64_t* bases, int64_t* ops) {
  Aligner* a = static_cast<Aligner*>(h);
  if (cells) *cells = a->ctr.cells;
  if (bases) *bases = a->ctr.bases;
  if (ops) *ops = a->ctr.ops;
}

// align_benchmark's per-pair dispatch and output, src/bin/align_benchmark.rs:466-504, 593-672
int32_t wfo_cli_line(void* h, int span, const int32_t* free4, int biwfa, int score_only,
                     const char* p, int32_t n, const char* t, int32_t m, char* out, int32_t cap) {
  Aligner* a = static_cast<Aligner*>(h);
  const uint8_t* P = (const uint8_t*)p;
  const uint8_t* T = (const uint8_t*)t;
  int32_t wfa_score;
  if (biwfa && span != 0) return -1;
  if (span == 0 && biwfa && score_only) wfa_score = a->align_biwfa_score(P, n, T, m);
  else if (span == 0 && biwfa) wfa_score = a->align_biwfa(P, n, T, m);
  else if (span == 0) wfa_score = a->align_end2end(P, n, T, m);
  else if (span == 1) wfa_score = a->align_endsfree(P, n, T, m);
  else {
    if (free4[0] > n || free4[1] > n || free4[2] > m || free4[3] > m) return -1;
    wfo_set_alignment_free_ends(h, free4[0], free4[1], free4[2], free4[3]);
    wfa_score = a->align_endsfree(P, n, T, m);
  }
  bool failed_bi = biwfa && score_only && a->status != COMPLETED;
  int32_t ev = n, eh = m;
  bool have_end_score = false;
  int32_t end_score = 0;
  bool unreached = a->status == PARTIAL || a->status == END_UNREACHABLE;
  if (!biwfa && unreached) {
    ev = wrap_sub(a->end_pos.offset, a->end_pos.k);
    eh = a->end_pos.offset;
    if (a->end_pos.score >= 0) { have_end_score = true; end_score = a->end_pos.score; }
  }
  if (have_end_score) wfa_score = end_score;
  int32_t outscore;
  const Penalties& pen = a->pen;
  // --no-c-compat: score-only output with no alignment behind it is -1
  // (src/bin/align_benchmark.rs:396-405, 641-652).
  const bool no_alignment =
      failed_bi || (!biwfa && unreached && a->end_pos.offset == OFFSET_NULL);
  if (score_only && a->compat == 1 && no_alignment) {
    outscore = -1;
  } else if (failed_bi) {
    outscore = INT32_MIN;
  } else if (!score_only) {
    const Cigar& c = a->cigar;
    if (c.empty()) outscore = -1;
    else if (pen.metric == EDIT || pen.metric == INDEL) outscore = c.score_edit();
    else if (pen.metric == LINEAR) outscore = c.score_gap_linear(pen.orig);
    else if (pen.metric == AFFINE) outscore = c.score_gap_affine(pen.orig);
    else outscore = c.score_gap_affine2p(pen.orig);
  } else {
    if (pen.metric == EDIT || pen.metric == INDEL) outscore = wfa_score;
    else if (pen.match_ < 0) outscore = pen.wf_score_to_sw_score(ev, eh, wfa_score);
    else outscore = -wfa_score;
  }
  std::string cg = (score_only || a->cigar.empty()) ? std::string("-") : a->cigar.rle();
  std::string line = std::to_string(outscore) + "\t" + cg;
  int32_t len = (int32_t)line.size();
  if (out && cap > 0) {
    int32_t c = std::min(len, cap - 1);
    std::memcpy(out, line.data(), (size_t)c);
    out[c] = 0;
  }
  return len;
}

double wfo_batch(int metric, const int32_t* pen, int compute_alignment, int mode, int hkind,
                 const int32_t* hp, const int32_t* free4, const char* seqs, const int64_t* p_off,
                 const int32_t* p_len, const int64_t* t_off, const int32_t* t_len, int64_t count,
                 int threads, int32_t* scores, int32_t* status, int64_t* cigar_hash,
                 int64_t* work3) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  std::atomic<int> ready{0};
  std::atomic<bool> go{false};
  std::vector<double> secs((size_t)threads, 0.0);
  std::vector<int64_t> work((size_t)threads * 3, 0);
  for (int tid = 0; tid < threads; ++tid) {
    pool.emplace_back([&, tid]() {
      Aligner* a = static_cast<Aligner*>(wfo_create(metric, pen));
      if (!a) { ready++; return; }
      wfo_set_alignment_scope(a, compute_alignment);
      if (hkind != H_NONE) wfo_set_heuristic(a, hkind, hp[0], hp[1], hp[2]);
      if (mode == 1) {
        if (free4) wfo_set_alignment_free_ends(a, free4[0], free4[1], free4[2], free4[3]);
        else wfo_set_alignment_extension(a);
      }
      ready++;
      while (!go.load()) std::this_thread::yield();
      auto t0 = std::chrono::steady_clock::now();
      for (int64_t i = tid; i < count; i += threads) {
        const uint8_t* P = (const uint8_t*)seqs + p_off[i];
        const uint8_t* T = (const uint8_t*)seqs + t_off[i];
        int32_t s;
        if (mode == 0) s = a->align_end2end(P, p_len[i], T, t_len[i]);
        else if (mode == 1) s = a->align_endsfree(P, p_len[i], T, t_len[i]);
        else s = a->align_biwfa(P, p_len[i], T, t_len[i]);
        if (scores) scores[i] = s;
        if (status) status[i] = a->status;
        if (work3) {
          work[(size_t)tid * 3] += a->ctr.cells;
          work[(size_t)tid * 3 + 1] += a->ctr.bases;
          work[(size_t)tid * 3 + 2] += a->ctr.ops;
        }
        if (cigar_hash) {
          uint64_t hsh = 1469598103934665603ull;
          const Cigar& c = a->cigar;
          if (compute_alignment || mode == 2)
            for (int64_t j = c.begin; j < c.end; ++j) hsh = (hsh ^ c.ops[(size_t)j]) * 1099511628211ull;
          cigar_hash[i] = (int64_t)hsh;
        }
      }
      secs[(size_t)tid] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      delete a;
    });
  }
  while (ready.load() < threads) std::this_thread::yield();
  auto w0 = std::chrono::steady_clock::now();
  go.store(true);
  for (auto& th : pool) th.join();
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  (void)secs;
  if (work3) {
    work3[0] = work3[1] = work3[2] = 0;
    for (int tid = 0; tid < threads; ++tid)
      for (int j = 0; j < 3; ++j) work3[j] += work[(size_t)tid * 3 + j];
  }
  return wall;
}

void wfo_hash_ops(const uint8_t* ops, const int64_t* begin, const int32_t* len, int64_t count,
                  int threads, int64_t* out) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int tid = 0; tid < threads; ++tid) {
    pool.emplace_back([=]() {
      for (int64_t i = tid; i < count; i += threads) {
        uint64_t hsh = 1469598103934665603ull;
        const uint8_t* c = ops + begin[i];
        for (int32_t j = 0; j < len[i]; ++j) hsh = (hsh ^ c[j]) * 1099511628211ull;
        out[i] = (int64_t)hsh;
      }
    });
  }
  for (auto& th : pool) th.join();
}

}  // extern "C"
