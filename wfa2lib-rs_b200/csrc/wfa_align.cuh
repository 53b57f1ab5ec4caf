// wfa_align.cuh -- the per-pair wavefront aligner run by one warp.
//
// One warp aligns one pair.  The control flow (score loop, input fetch,
// range union, null steps, termination, heuristics, backtrace) is
// warp-uniform: every lane holds the same scalar state.  Lanes split the
// diagonals of each wavefront (k = lo + lane, lo + lane + 32, ...) and meet in
// warp reductions for the trims, termination and heuristic cutoffs.
//
// Storage model.  The reference keeps, per wavefront, an allocation, limits
// [lo, hi] and an initialised range, and NULL-fills input ends before reading
// them (src/wavefront.rs:422-457).  Every cell outside the initialised range
// reads as OFFSET_NULL there, so here a wavefront stores exactly its
// initialised range [a, b] and a read outside it returns OFFSET_NULL
// directly; no fill is ever written.  Limits and the initialised range evolve
// as in the reference: both set by the compute step and trim_ends; limits
// narrowed by the heuristics; the range emptied when a cutoff empties the
// wavefront.  Component slots are a ring of max_score_scope scores; in
// high-memory (CIGAR) mode the M wavefronts of every score are also kept in a
// per-warp history arena for the backtrace.
//
// The same source compiles as host C++ with a one-lane "warp" (WFA_EMU):
// the CPU tests run that build against the oracle to check this logic before
// it runs on a GPU.  It is test-only and never part of the product library.
#pragma once

#include <stdint.h>

#include "wfa_common.h"

#if defined(__CUDACC__) && !defined(WFA_EMU)
#define WFA_D __device__ __forceinline__
#define WFA_DN __device__ __noinline__
#define WFA_WARP 32
#define WFA_CUDA_WARP 1
#else
#include <algorithm>
#include <climits>
#include <cstdlib>
#ifndef __CUDACC__
struct int4 { int x, y, z, w; };
struct int2 { int x, y; };
struct uint2 { unsigned x, y; };
#endif
#define WFA_D inline
#define WFA_DN inline
#ifdef WFA_EMU_THREADS
#include <barrier>
// Lanes of the emulated warp (32; 8 emulates an 8-lane group of the kernel).
#ifndef WFA_EMU_LANES
#define WFA_EMU_LANES 32
#endif
#define WFA_WARP WFA_EMU_LANES
#else
#define WFA_WARP 1
#endif
#endif

namespace wfab {

// Index checks of the aligner's invariants.  The emulation builds abort on a
// failed check; the device-checks build (WFA_DEVICE_CHECKS) counts it in
// P.check_count and takes the given way out (skip the access, or stop the
// pair with a retry) so that no access goes out of bounds; the product build
// compiles them out.
#if !(defined(__CUDACC__) && !defined(WFA_EMU))
#define WFA_CHECK(cond, on_fail) \
  do {                          \
    if (!(cond)) std::abort();  \
  } while (0)
#elif defined(WFA_DEVICE_CHECKS)
#define WFA_CHECK(cond, on_fail)                          \
  do {                                                    \
    if (!(cond)) {                                        \
      if (P.check_count) atomicAdd(P.check_count, 1);     \
      on_fail;                                            \
    }                                                     \
  } while (0)
#else
#define WFA_CHECK(cond, on_fail) \
  do {                          \
  } while (0)
#endif

// ---------------------------------------------------------------------------
// Warp primitives (one-lane stand-ins in the emulation build)
// ---------------------------------------------------------------------------
#if defined(WFA_EMU_THREADS)
// Test-only: WFA_WARP host threads play the lanes of one warp (or lane
// group); __syncwarp and the warp reductions become barriers, so lane
// partitioning, reductions and warp-uniform control flow are exercised
// exactly as on the GPU.
struct EmuWarp {
  std::barrier<> bar{WFA_WARP};
  int red[WFA_WARP];
};
extern thread_local int g_emu_lane;
extern EmuWarp* g_emu_warp;
#endif

struct Warp {
#if defined(WFA_EMU_THREADS)
  static int lane() { return g_emu_lane; }
  static void sync() { g_emu_warp->bar.arrive_and_wait(); }
  static int reduce(int v, bool mx) {
    EmuWarp* w = g_emu_warp;
    w->red[g_emu_lane] = v;
    w->bar.arrive_and_wait();
    int r = w->red[0];
    for (int i = 1; i < WFA_WARP; ++i) r = mx ? (w->red[i] > r ? w->red[i] : r) : (w->red[i] < r ? w->red[i] : r);
    w->bar.arrive_and_wait();
    return r;
  }
  static int min(int v) { return reduce(v, false); }
  static int max(int v) { return reduce(v, true); }
  static unsigned any(bool p) { return (unsigned)reduce(p ? 1 : 0, true); }
  // Lanes below this one with p set; *total: lanes with p set.
  static int rank(bool p, int* total) {
    EmuWarp* w = g_emu_warp;
    w->red[g_emu_lane] = p ? 1 : 0;
    w->bar.arrive_and_wait();
    int below = 0, all = 0;
    for (int i = 0; i < WFA_WARP; ++i) { all += w->red[i]; if (i < g_emu_lane) below += w->red[i]; }
    w->bar.arrive_and_wait();
    *total = all;
    return below;
  }
  static uint32_t atomic_or(uint32_t* a, uint32_t v) { return __atomic_fetch_or(a, v, __ATOMIC_RELAXED); }
  static int popc(uint32_t x) { return __builtin_popcount(x); }
  static uint32_t ffs(uint32_t x) { return x ? (uint32_t)__builtin_ctz(x) + 1 : 0; }
  static uint32_t clz(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32; }
  static uint32_t funnel(uint32_t lo, uint32_t hi, uint32_t s) {
    s &= 31;
    uint64_t v = ((uint64_t)hi << 32) | lo;
    return (uint32_t)(v >> s);
  }
#elif WFA_WARP == 32
  static WFA_D int lane() { return threadIdx.x & 31; }
  static WFA_D int min(int v) { return __reduce_min_sync(0xffffffffu, v); }
  static WFA_D int max(int v) { return __reduce_max_sync(0xffffffffu, v); }
  static WFA_D unsigned any(bool p) { return __ballot_sync(0xffffffffu, p); }
  static WFA_D void sync() { __syncwarp(); }
  static WFA_D int popc(uint32_t x) { return __popc(x); }
  static WFA_D uint32_t ffs(uint32_t x) { return (uint32_t)__ffs((int)x); }
  static WFA_D uint32_t clz(uint32_t x) { return (uint32_t)__clz((int)x); }
  static WFA_D uint32_t funnel(uint32_t lo, uint32_t hi, uint32_t s) { return __funnelshift_r(lo, hi, s); }
#else
  static int lane() { return 0; }
  static int min(int v) { return v; }
  static int max(int v) { return v; }
  static unsigned any(bool p) { return p ? 1u : 0u; }
  static int rank(bool p, int* total) { *total = p ? 1 : 0; return 0; }
  static uint32_t atomic_or(uint32_t* a, uint32_t v) { uint32_t o = *a; *a = o | v; return o; }
  static int popc(uint32_t x) { return __builtin_popcount(x); }
  static void sync() {}
  static uint32_t ffs(uint32_t x) { return x ? (uint32_t)__builtin_ctz(x) + 1 : 0; }
  static uint32_t clz(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32; }
  static uint32_t funnel(uint32_t lo, uint32_t hi, uint32_t s) {
    s &= 31;
    uint64_t v = ((uint64_t)hi << 32) | lo;
    return (uint32_t)(v >> s);
  }
#endif
};

// A group of LW lanes that aligns one pair: LW = 32 is the whole warp; 4, 8
// or 16 put 8, 4 or 2 pairs in a warp (short pairs, whose wavefronts are a
// few diagonals wide).  The groups of a warp run the same code on different
// pairs; every collective names only the group's own lanes.  LW = 64, 128,
// 256 or 512 is a team of LW / 32 whole warps, the whole block (long pairs,
// whose wavefronts are thousands of diagonals wide): its collectives meet at
// named barrier 1 (barrier 0 is __syncthreads) and combine the warps'
// partial results in shared memory.
// A barrier also orders the team's shared- and global-memory accesses, as
// __syncwarp does a warp's.  In the emulation builds the emulated warp is
// the group.
#if defined(WFA_CUDA_WARP)
template <int LW>
struct Lanes {
  static_assert(LW == 4 || LW == 8 || LW == 16 || LW == 32 || LW == 64 || LW == 128 || LW == 256 ||
                    LW == 512,
                "lane group width");
  static constexpr bool TEAM = LW > 32;
  static constexpr int NW = TEAM ? LW / 32 : 1;  // warps of a team
  static WFA_D unsigned mask() {
    return LW >= 32 ? 0xffffffffu : ((1u << LW) - 1u) << ((threadIdx.x & 31) & ~(LW - 1));
  }
  static WFA_D int lane() { return threadIdx.x & (LW - 1); }
  static WFA_D void sync() {
    if constexpr (TEAM) {
      // The warp's lanes may reach this point apart (after lane-dependent
      // branches): reconverge them first, and use the barrier form that does
      // not assume a converged warp (bar.sync is barrier.sync.aligned).
      __syncwarp();
      asm volatile("barrier.sync 1, %0;" ::"n"(LW) : "memory");
    } else {
      __syncwarp(mask());
    }
  }
  // One partial per warp of the block: up to 16 warps (512 threads).
  static WFA_D int* partials() {
    __shared__ int part[16];
    return part;
  }
  static WFA_D int team_first_warp() { return (int)(threadIdx.x >> 5) & ~(NW - 1); }
  // The warps' partials of a team, combined after a barrier; a second
  // barrier keeps the next collective from overwriting them early.
  static WFA_D int min(int v) {
    const int w = __reduce_min_sync(mask(), v);
    if constexpr (!TEAM) {
      return w;
    } else {
      int* part = partials();
      if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = w;
      sync();
      const int b = team_first_warp();
      int r = part[b];
#pragma unroll
      for (int i = 1; i < NW; ++i) r = ::min(r, part[b + i]);
      sync();
      return r;
    }
  }
  static WFA_D int max(int v) {
    const int w = __reduce_max_sync(mask(), v);
    if constexpr (!TEAM) {
      return w;
    } else {
      int* part = partials();
      if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = w;
      sync();
      const int b = team_first_warp();
      int r = part[b];
#pragma unroll
      for (int i = 1; i < NW; ++i) r = ::max(r, part[b + i]);
      sync();
      return r;
    }
  }
  static WFA_D unsigned any(bool p) {
    if constexpr (!TEAM) return __ballot_sync(mask(), p) & mask();
    else return (unsigned)max(p ? 1 : 0);
  }
  // Lanes of the group below this one with p set; *total: the group's lanes
  // with p set.
  static WFA_D int rank(bool p, int* total) {
    const unsigned b = __ballot_sync(mask(), p) & mask();
    const int below = __popc(b & ((1u << (threadIdx.x & 31)) - 1u));
    if constexpr (!TEAM) {
      *total = __popc(b);
      return below;
    } else {
      int* part = partials();
      if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = __popc(b);
      sync();
      const int f = team_first_warp(), me = (int)(threadIdx.x >> 5);
      int tot = 0, before = 0;
#pragma unroll
      for (int i = 0; i < NW; ++i) {
        const int c = part[f + i];
        before += f + i < me ? c : 0;
        tot += c;
      }
      sync();
      *total = tot;
      return before + below;
    }
  }
  static WFA_D uint32_t atomic_or(uint32_t* a, uint32_t v) { return atomicOr(a, v); }
};
#else
template <int LW>
struct Lanes : Warp {
  static_assert(LW == WFA_WARP, "the emulated warp is the lane group");
};
#endif

WFA_D int imin(int a, int b) { return a < b ? a : b; }
WFA_D int imax(int a, int b) { return a > b ? a : b; }
WFA_D int64_t lmax(int64_t a, int64_t b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// Sequences.  fetch(pos) returns the UNITS codes starting at pos, lowest code
// in the lowest bits; positions outside [0, len) hold unspecified codes, and
// callers clamp to the sequence lengths (the reference's sentinels end every
// extension at the end of either sequence, src/sequences.rs:12-19).
// ---------------------------------------------------------------------------
struct SeqPacked {  // 2-bit codes, 16 per word; a view may start at base `off` of w
  static constexpr int UNITS = 16, BITS = 2;
  const uint32_t* w;
  int32_t len, nw;
  int32_t off = 0;
  WFA_D uint32_t word(int i) const { return (i >= 0 && i < nw) ? w[i] : 0u; }
  WFA_D uint32_t fetch(int pos) const {
    pos += off;
    if (pos < 0) {
      int s = -pos;
      return s >= 16 ? 0u : (word(0) << (2 * s));
    }
    int i = pos >> 4;
    return Warp::funnel(word(i), word(i + 1), (uint32_t)(2 * (pos & 15)));
  }
};

struct SeqAscii {  // bytes, any alignment
  static constexpr int UNITS = 4, BITS = 8;
  const uint8_t* p;
  int32_t len;
  // Aligned 32-bit word i relative to the word containing p[0]; loaded only
  // if it holds at least one byte of the sequence.
  WFA_D uint32_t word_at(int64_t i) const {
    uintptr_t a0 = ((uintptr_t)p) & ~(uintptr_t)3;
    uintptr_t a = a0 + (uintptr_t)(i * 4);
    uintptr_t end = (uintptr_t)p + (uintptr_t)len;
    if (i < 0 || len <= 0 || a >= end) return 0u;
    return *(const uint32_t*)a;
  }
  WFA_D uint32_t fetch(int pos) const {
    int sh = 0;
    if (pos < 0) {
      sh = -pos;
      if (sh >= 4) return 0u;
      pos = 0;
    }
    uintptr_t off = (((uintptr_t)p) & 3) + (uintptr_t)pos;
    int64_t i = (int64_t)(off >> 2);
    return Warp::funnel(word_at(i), word_at(i + 1), (uint32_t)(8 * (off & 3))) << (8 * sh);
  }
};

// Matches of P[v..] with T[h..], at most R (forward extension).
template <class S>
WFA_D int lcp_fwd(const S& P, int v, const S& T, int h, int R) {
  int l = 0;
  while (l < R) {
    uint32_t x = P.fetch(v + l) ^ T.fetch(h + l);
    if (x) { l += (int)((Warp::ffs(x) - 1) / S::BITS); break; }
    l += S::UNITS;
  }
  return l < R ? l : R;
}

// Matches ending at P[v-1], T[h-1] walking backwards, at most R
// (st_backward_matches, src/backtrace.rs:668-686).
template <class S>
WFA_D int lcp_bwd(const S& P, int v, const S& T, int h, int R) {
  int l = 0;
  while (l < R) {
    uint32_t x = P.fetch(v - l - S::UNITS) ^ T.fetch(h - l - S::UNITS);
    if (x) { l += (int)(Warp::clz(x) / S::BITS); break; }
    l += S::UNITS;
  }
  return l < R ? l : R;
}

// ---------------------------------------------------------------------------
// Wavefront descriptors
// ---------------------------------------------------------------------------
constexpr int kPresent = 1, kNullFlag = 2;
// Packed CIGARs of the med/low (piggyback) backtrace, src/pcigar.rs:13-35:
// up to 16 two-bit operations per u32, pushed at the low end.
constexpr uint32_t kPcDel = 1, kPcMisms = 2, kPcIns = 3;
constexpr uint32_t kPcFullMask = 0x40000000u, kPcAlmostFullMask = 0x10000000u, kPcHalfFullMask = 0x00010000u;
constexpr int kPcMaxLength = 16;
constexpr uint32_t kBtNull = 0xFFFFFFFFu;  // BT_BLOCK_IDX_NULL, src/bt_buffer.rs:11
WFA_D uint32_t pc_push(uint32_t pc, uint32_t op) { return (pc << 2) | op; }
constexpr int32_t kAdUnknown = INT32_MAX / 4, kAdNone = INT32_MIN / 4;
constexpr int CM = 0, CI1 = 1, CD1 = 2, CI2 = 3, CD2 = 4;

struct WfD {
  int32_t* vals;  // cell k at vals[k - a]
  int32_t lo, hi; // limits
  int32_t a, b;   // initialised range
  int32_t flags;
  // Upper bound on the antidiagonal 2 * offset - k of the stored cells
  // (kAdUnknown: none known).  BiWFA's breakpoint scans skip wavefront
  // pairs whose bounds cannot add up to a meeting.
  int32_t adub;
};

WFA_D bool wf_present(const WfD& d) { return (d.flags & kPresent) != 0; }
WFA_D bool wf_is_null(const WfD& d) { return !(d.flags & kPresent) || (d.flags & kNullFlag); }
WFA_D WfD wf_none() {
  WfD d;
  d.vals = nullptr; d.lo = 1; d.hi = -1; d.a = 1; d.b = 0; d.flags = 0; d.adub = kAdUnknown;
  return d;
}
// Cell read with the reference's semantics (OFFSET_NULL outside the
// initialised range; null inputs read as the null wavefront).
WFA_D int32_t rd(const WfD& d, int k) {
  return (k >= d.a && k <= d.b) ? d.vals[k - d.a] : kOffsetNull;
}
// Antidiagonal bound of a live wavefront (kAdNone for an absent or null one).
WFA_D int32_t ad_of(const WfD& d) {
  return (d.flags == kPresent) ? d.adub : kAdNone;
}
WFA_D bool cell_in_bounds(int32_t off, int k, int n, int m) {
  return (uint32_t)off <= (uint32_t)m && (uint32_t)(off - k) <= (uint32_t)n;
}

// Heuristic state, src/heuristic.rs:62-148.
struct HState {
  int32_t steps_wait, max_sw_score, max_wf_score, max_sw_k, max_sw_off, zdrop_last;
};

// Per-warp workspace pointers.
struct Workspace {
  WfD* ring;        // [scope][NC] descriptors (shared memory on the GPU)
  int32_t* ringv;   // [scope][NC][wmax] cells
  int4* hist;       // [hist_scores] M history records {a, b, cell offset of a, present}
  int32_t* harena;  // M history cells
  int32_t* dom;     // Corrected-mode dominance array (NC x diagonals), or null
  int32_t* ringg;   // compact ring: rows wider than the ring's slots (device memory), or null
  // Med/low: the backtrace buffer (blocks {pcigar, prev}), the initial
  // positions of its chains ({v, h}) and the mark bitmap of its compaction.
  uint2* bt;
  int2* btinit;
  uint32_t* btmark;
};

// GEN = false compiles the common configuration only (end-to-end, no
// heuristic): the ends-free and heuristic code paths drop out, which keeps
// the kernel body small.  UNR diagonals per lane per pass of the affine
// compute and of the BiWFA extend: their loads are all issued before any
// result is stored, so a lane keeps UNR cells' loads in flight (wide
// wavefronts of long pairs, whose cells live in device memory).
// PB: the med/low (piggyback) code is compiled in (a separate kernel: it
// would otherwise cost the other general alignments registers).
template <int CLS, class S, bool GEN = true, int UNR = 1, int LW = WFA_WARP, bool PB = false>
struct PairAligner {
  using G = Lanes<LW>;
  static constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  static constexpr bool AFF = CLS >= kAffineClass;
  static constexpr bool TWO = CLS == kAffine2pClass;

  const AlignParams& P;
  Workspace ws;
  S pat, txt;
  int32_t n, m;
  int32_t lane;
  int32_t scope, wmax;
  // Compact cell ring (the unidirectional aligner; BiWFA's overlap scans read
  // every slot of the scope, so its rings keep one slot per score): a
  // component's cells are only read within a fixed number of scores after
  // they are written (M at s + x, s + o + e; a gap component at s + e), and
  // only scores that are multiples of gstep hold wavefronts, so each
  // component gets a round-robin ring of depth (its longest read offset /
  // gstep) + 1, a new slot per wavefront it stores.  Rows wider than wmax go
  // to the same slot of a second ring of width P.wspill in device memory.
  // The launch provides P.ring_slots slots per lane group (0: this layout is
  // off).  I and D of a piece are always stored together, so they share one
  // slot counter (advanced by D's allocation).
  bool compact = false;
  int16_t dm = 0, d1 = 0, d2 = 0;  // depths: M, I1/D1, I2/D2
  int16_t nm = 0, n1 = 0, n2 = 0;  // next slots: M, piece 1, piece 2
  bool modular;  // score-only: no M history
  // BiWFA growth phase (breakpoint searches before their overlap scans):
  // nothing reads an I/D row more than e scores old, so the I/D rows go to
  // a ring of e + 1 rows per component after the scope x NC rows
  // (bi_idc_rows), which keeps a search's footprint near M's alone.
  bool idc = false;
  int32_t cap;   // num_wavefronts score cap (high memory)
  int32_t p0, pf, t0, tf;
  bool endsfree;
  int32_t hist_lo, hist_hi;
  // Heuristic (the aligner's own copy: BiWFA shifts the band per sub-problem).
  int32_t hkind, hp0, hp1, hp2;
  // History components (1: M only, for Singletrack / linear; NC: all, for the
  // classic affine backtrace of the BiWFA base case) and whether all-null
  // steps store null slots (BiWFA's overlap scans read every ring slot).
  int32_t hist_nc;
  bool keep_null_slots;
  // Med/low memory with an alignment: the piggyback backtrace as the
  // reference runs it (src/compute/piggyback.rs).  Every cell of every
  // component carries a packed CIGAR and the index of the backtrace-buffer
  // block it continues, stored pcoff and 2 * pcoff words after the cell's
  // offset in the same ring slot; full packed CIGARs move into the buffer
  // (ws.bt, bt_used of P.bt_cap blocks) and chains start at initial blocks
  // whose positions are in ws.btinit.  There is no history: med/low needs
  // only the ring and the buffer.  The occupancy the offload tracks
  // (bt_occupancy_max) rides in a wavefront's descriptor, in adub.
  bool pgb = false;
  int64_t pcoff = 0;
  int32_t bt_used = 0, bi_used = 0;
  int32_t mL = 1, mH = 0;  // the cells the current score's M kernel wrote
  uint32_t cand_pc = 0, cand_pv = kBtNull, zd_pc = 0, zd_pv = kBtNull;
  // Compat::Corrected ends-free with a match reward (src/aligner.rs:1104-1345):
  // the end candidate (the best cell reaching a free end so far, its total
  // score) and the begin-free dominance array (ws.dom, NC x diagonals from
  // hist_lo, the furthest offset each diagonal reached at an earlier score).
  bool corr = false, dom_on = false;
  bool c_has = false;
  int32_t c_total = 0, c_score = 0, c_k = 0, c_off = 0;
  int32_t dom_len = 0;
  int32_t comp_end;  // component whose end diagonal terminates (BiWFA), else M
  int32_t cscore, cidx;  // current score and its ring index
  // Scores that are not multiples of gstep can have no wavefront: every input
  // score differs from them by a multiple of gstep (the gcd of the score
  // offsets the recurrences use, and of the begin-free seed scores).  Their
  // steps are the reference's all-null steps; only the null-step count moves.
  int32_t gstep, gphase;
  int32_t num_null_steps;
  int32_t status;
  int32_t end_score, end_k, end_off;
  HState hs;
  bool retry;
  int64_t hused;
  // CIGAR (written backwards into the pair's slot)
  uint8_t* cg;
  int64_t cg_cap, cg_begin, cg_end;
  int32_t cg_score, cg_ev, cg_eh;

  WFA_D PairAligner(const AlignParams& p) : P(p) {}
  WFA_D int hk() const { return GEN ? hkind : (int)WFA_HEURISTIC_NONE; }
  WFA_D bool ef() const { return GEN && endsfree; }

  // ---- slots --------------------------------------------------------------
  // Descriptor ring index of score t (cscore - scope < t <= cscore), kept
  // without a division: cidx == (cscore >> gshift) % dscope is advanced with
  // the score loop.  With the compact layout and a power-of-two score step
  // (gshift > 0) only scores that are multiples of it have slots, and t must
  // be one of them; otherwise every score has one (dscope == scope).
  int32_t gshift = 0, dscope = 0;
  WFA_D int sidx(int t) const {
    int i = cidx - ((cscore - t) >> gshift);
    i = i < 0 ? i + dscope : i;
    WFA_CHECK(i >= 0 && i < dscope, i = 0);
    return i;
  }
  WFA_D void advance() {
    ++cscore;
    if ((cscore & ((1 << gshift) - 1)) == 0) cidx = cidx + 1 == dscope ? 0 : cidx + 1;
  }
  WFA_D WfD& slot(int c, int s) { return ws.ring[sidx(s) * NC + c]; }
  // Slot (c, s) holds a live wavefront: present and not null (flags are
  // 0 none, kPresent, or kPresent|kNullFlag).
  WFA_D bool live(int c, int s) { return s >= 0 && slot(c, s).flags == kPresent; }
  WFA_D WfD get(int c, int s) {  // input fetch (score may be negative)
    if (s < 0) return wf_none();
    return slot(c, s);
  }
  // Descriptor stores are made by lane 0; callers reach a warp-collective
  // operation (or an explicit sync) between reading a slot and storing into
  // it, and sync() makes the stores visible before the next step reads them.
  WFA_D void put_ns(int c, int s, const WfD& d) {
    if (lane == 0) slot(c, s) = d;
  }
  WFA_D void put(int c, int s, const WfD& d) {
    put_ns(c, s, d);
    G::sync();
  }
  // Storage for an output of component c at score s covering [L, H]
  // (s is always the current score).
  WFA_D int32_t* alloc(int c, int s, int L, int H) {
    int64_t w = (int64_t)H - L + 1;
    int64_t idx;
    if (compact) {
      if (c == CM) {
        idx = nm;
        nm = nm + 1 == dm ? 0 : nm + 1;
      } else if (c == CI1 || c == CD1) {
        idx = dm + (c == CD1 ? d1 : 0) + n1;
        if (c == CD1) n1 = n1 + 1 == d1 ? 0 : n1 + 1;
      } else {
        idx = dm + 2 * d1 + (c == CD2 ? d2 : 0) + n2;
        if (c == CD2) n2 = n2 + 1 == d2 ? 0 : n2 + 1;
      }
    } else if (idc && c != CM) {
      const int r1 = P.e1 + 1, r2 = P.e2 + 1;
      const int depth = (c == CI1 || c == CD1) ? r1 : r2;
      const int first = c == CI1 ? 0 : c == CD1 ? r1 : c == CI2 ? 2 * r1 : 2 * r1 + r2;
      idx = (int64_t)scope * NC + first + s % depth;
    } else {
      idx = (int64_t)sidx(s) * NC + c;
    }
    WFA_CHECK(!compact || idx < P.ring_slots, { retry = true; return nullptr; });
    WFA_CHECK(compact || idx < (int64_t)scope * NC + (modular ? bi_idc_rows(NC, P.e1, P.e2) : 0),
              { retry = true; return nullptr; });
    if (w <= wmax) {
      int32_t* base = ws.ringv + idx * wmax;
      if (PB && pgb && c == CM) { mbase = base; mL = L; mH = H; }
      return base;
    }
    if (compact && ws.ringg && w <= P.wspill) return ws.ringg + idx * P.wspill;
    retry = true;
    return nullptr;
  }

  // ---- med/low: packed CIGARs and the backtrace buffer -----------------------
  int32_t* mbase = nullptr;  // the current score's M slot (cells from mL)
  WFA_D uint32_t* pcs(int32_t* v) const { return reinterpret_cast<uint32_t*>(v + pcoff); }
  WFA_D uint32_t* pvs(int32_t* v) const { return reinterpret_cast<uint32_t*>(v + 2 * pcoff); }
  // (pcigar, prev) of cell k as the kernels read it: zero outside the
  // initialised range (init_ends zeroes them, src/wavefront.rs:422-457, and
  // the null wavefront holds zeroes).
  WFA_D uint32_t rpc(const WfD& d, int k) const { return (k >= d.a && k <= d.b) ? pcs(d.vals)[k - d.a] : 0u; }
  WFA_D uint32_t rpv(const WfD& d, int k) const { return (k >= d.a && k <= d.b) ? pvs(d.vals)[k - d.a] : 0u; }
  // bt_occupancy_max of an input (0 if absent or null).
  WFA_D int32_t occ_of(const WfD& d) const { return d.flags == kPresent ? d.adub : 0; }
  // bt_or_zero (src/wavefront.rs:410-416) on the current score's M: the
  // cells its kernel wrote (mL..mH), else zeroes.
  WFA_D void m_bt(int k, uint32_t& c, uint32_t& v) const {
    if (mbase && k >= mL && k <= mH) { c = pcs(mbase)[k - mL]; v = pvs(mbase)[k - mL]; }
    else { c = 0; v = 0; }
  }
  // init_block (src/bt_buffer.rs:134-139) for the cell at base[i]: an empty
  // pcigar continuing a new initial block at (v, h) (set_bt_init,
  // src/aligner.rs:213-225).  Lane 0 writes.
  WFA_D void bt_init_cell(int32_t* base, int64_t i, int v, int h) {
    if (bt_used >= P.bt_cap || bi_used >= P.bt_init_cap) { retry = true; return; }
    if (lane == 0) {
      ws.btinit[bi_used] = int2{v, h};
      ws.bt[bt_used] = uint2{(uint32_t)bi_used, kBtNull};
      pcs(base)[i] = 0;
      pvs(base)[i] = (uint32_t)bt_used;
    }
    ++bi_used;
    ++bt_used;
  }
  // zero_bt (src/wavefront.rs:570-580) on cells base[i0 .. i1].
  WFA_D void bt_zero(int32_t* base, int64_t i0, int64_t i1) {
    for (int64_t i = i0 + lane; i <= i1; i += LW) { pcs(base)[i] = 0; pvs(base)[i] = 0; }
  }
  // offload_blocks_selective (src/compute/piggyback.rs:530-555) on output
  // cells [lo, hi] of a slot whose cells start at L: every live cell whose
  // pcigar is at or above `mask` moves into a new block (in ascending k, as
  // the reference numbers them) and continues from it.
  WFA_D void offload_cells(int32_t* base, int L, int lo, int hi, uint32_t mask) {
    uint32_t* pc = pcs(base);
    uint32_t* pv = pvs(base);
    for (int k0 = lo; k0 <= hi; k0 += LW) {
      const int k = k0 + lane;
      bool mv = false;
      uint32_t c = 0;
      if (k <= hi) {
        c = pc[k - L];
        mv = base[k - L] >= 0 && c >= mask;
      }
      int total;
      const int r = G::rank(mv, &total);
      if (bt_used + total > P.bt_cap) { retry = true; return; }
      if (mv) {
        ws.bt[bt_used + r] = uint2{c, pv[k - L]};
        pc[k - L] = 0;
        pv[k - L] = (uint32_t)(bt_used + r);
      }
      bt_used += total;
    }
    G::sync();
  }
  WFA_D bool pb_low() const { return P.piggyback == 2; }
  // offload_blocks_linear / _affine (:557-585); returns the occupancy left.
  WFA_D int32_t offload_linear_cells(int32_t* base, int L, int lo, int hi) {
    offload_cells(base, L, lo, hi, pb_low() ? kPcFullMask : kPcHalfFullMask);
    return pb_low() ? kPcMaxLength - 1 : kPcMaxLength / 2;
  }
  WFA_D int32_t offload_affine_cells(int32_t* base, int L, int lo, int hi) {
    offload_cells(base, L, lo, hi, pb_low() ? kPcAlmostFullMask : kPcHalfFullMask);
    return pb_low() ? kPcMaxLength - 2 : kPcMaxLength / 2;
  }
  // occupancy of a gap component fed by an M opening and its own extension
  // (:611-620).
  WFA_D int32_t occ_gap(const WfD& open, const WfD& ext) const {
    int32_t o = open.flags == kPresent ? open.adub + 1 : 0;
    if (ext.flags == kPresent) o = imax(o, ext.adub + 1);
    return o;
  }
  // offload_affine_component (:622-632) for an output with occupancy occ.
  WFA_D int32_t offload_component(int32_t* base, int L, int lo, int hi, int32_t occ) {
    return occ >= kPcMaxLength - 1 ? offload_affine_cells(base, L, lo, hi) : occ;
  }
  // Depths of the compact ring for score step gstep (the longest read offset
  // of M is scope - 1; of a gap component its extension penalty).
  WFA_D void compact_depths() {
    dm = (int16_t)((scope - 1) / gstep + 1);
    d1 = (int16_t)(AFF ? P.e1 / gstep + 1 : 0);
    d2 = (int16_t)(TWO ? P.e2 / gstep + 1 : 0);
    nm = n1 = n2 = 0;
    if (dm + 2 * d1 + 2 * d2 > P.ring_slots) retry = true;
  }
  // High memory: once M at score s is final (after its extend step), copy its
  // initialised range to the history arena for the backtrace.
  WFA_D void hist_commit(int s) {
    if (modular || (PB && pgb)) return;
    if ((int64_t)(s + 1) * hist_nc > P.hist_scores) { retry = true; return; }
    for (int c = 0; c < hist_nc; ++c) {
      WfD d = slot(c, s);
      int4 r;
      r.x = d.a; r.y = d.b; r.z = 0; r.w = 0;
      if (wf_present(d)) {
        int64_t w = d.b >= d.a ? (int64_t)d.b - d.a + 1 : 0;
        if (hused + w > P.hist_words) { retry = true; return; }
        for (int64_t i = lane; i < w; i += LW) ws.harena[hused + i] = d.vals[i];
        r.z = (int32_t)hused;
        r.w = 1;
        hused += w;
      }
      if (lane == 0) ws.hist[(int64_t)s * hist_nc + c] = r;
    }
    // No sync: the history is read only by the backtrace, which starts with one.
  }

  // ---- helpers --------------------------------------------------------------
  // num_wavefronts, src/components.rs:435-505 (components start sized for
  // 1000 x 1000, src/aligner.rs:377-378, and only grow).
  WFA_D int32_t dims_num(int32_t pl, int32_t tl) const {
    int32_t ad = pl > tl ? pl - tl : tl - pl, mn = imin(pl, tl);
    switch (CLS) {
      case kEditClass:
        return P.metric == WFA_METRIC_INDEL ? pl + tl + 1 : imax(pl, tl) + 1;
      case kLinearClass:
        return mn * P.mismatch + P.o1 * ad + 1;
      case kAffineClass:
        return mn * P.mismatch + P.o1 + ad * P.e1 + 1;
      default:
        return mn * P.mismatch + imin(P.o1 + ad * P.e1, P.o2 + ad * P.e2) + 1;
    }
  }
  WFA_D bool has_slot(int s) const { return modular || s < cap; }

  // endsfree_begin_k, src/aligner.rs:3408-3421
  WFA_D bool begin_k(int s, int& k) const {
    if (P.match == 0 || !ef()) return false;
    if (t0 == 0 && p0 == 0) return false;
    if (s % (-P.match) != 0) return false;
    k = s / (-P.match);
    return t0 >= k || p0 >= k;
  }

  WFA_D void clamp_band(int& lo, int& hi) const {  // src/aligner.rs:3308-3317
    if (hk() == WFA_HEURISTIC_BANDED_STATIC || hk() == WFA_HEURISTIC_BANDED_ADAPTIVE) {
      lo = imax(lo, hp0);
      hi = imin(hi, hp1);
    }
  }

  // Trim an output wavefront computed over [lo, hi] (trim_ends,
  // src/compute/mod.rs:14-49) given the warp's min/max in-bounds diagonal.
  WFA_D WfD finish(int32_t* base, int L, int lo, int hi, int vmin, int vmax) {
    WfD d;
    d.flags = kPresent;
    d.adub = kAdUnknown;
    if (vmax >= vmin && vmax != INT_MIN) {
      d.lo = vmin; d.hi = vmax;
    } else {
      d.lo = lo; d.hi = lo - 1;
      d.flags |= kNullFlag;
    }
    d.a = d.lo; d.b = d.hi;
    d.vals = base + (d.a - L);
    return d;
  }

  // Trim pass over stored cells [lo, hi] (used after endsfree_init).
  WFA_D WfD trim_pass(int32_t* base, int L, int lo, int hi) {
    int vmin = INT_MAX, vmax = INT_MIN;
    G::sync();
    for (int k = lo + lane; k <= hi; k += LW) {
      if (cell_in_bounds(base[k - L], k, n, m)) { vmin = imin(vmin, k); vmax = imax(vmax, k); }
    }
    vmin = G::min(vmin);
    vmax = G::max(vmax);
    return finish(base, L, lo, hi, vmin, vmax);
  }

  // endsfree_init, src/aligner.rs:3426-3452, on M stored at base (cell L)
  // and computed over [lo, hi]; returns the new limits through lo/hi.
  WFA_D void endsfree_init(int32_t* base, int L, int& lo, int& hi, int k) {
    G::sync();
    const bool bt = PB && pgb;  // seeds start chains (endsfree_init_offset, :3421-3434)
    if (t0 >= k) {
      if (hi >= k) {
        if (base[k - L] <= k) {
          G::sync();
          if (lane == 0) base[k - L] = k;
          if (bt) bt_init_cell(base, k - L, 0, k);
        }
      } else {
        for (int kk = hi + 1 + lane; kk < k; kk += LW) base[kk - L] = kOffsetNull;
        if (bt) bt_zero(base, hi + 1 - L, k - 1 - L);
        if (lane == 0) base[k - L] = k;
        if (bt) bt_init_cell(base, k - L, 0, k);
        hi = k;
      }
    }
    G::sync();
    if (p0 >= k) {
      if (lo <= -k) {
        if (base[-k - L] <= 0) {
          G::sync();
          if (lane == 0) base[-k - L] = 0;
          if (bt) bt_init_cell(base, -k - L, k, 0);
        }
      } else {
        if (lane == 0) base[-k - L] = 0;
        if (bt) bt_init_cell(base, -k - L, k, 0);
        for (int kk = -k + 1 + lane; kk < lo; kk += LW) base[kk - L] = kOffsetNull;
        if (bt) bt_zero(base, -k + 1 - L, lo - 1 - L);
        lo = -k;
      }
    }
    G::sync();
  }

  // endsfree_null_m, src/aligner.rs:3470-3494
  WFA_D WfD endsfree_null_m(int s, int k) {
    bool text = t0 >= k, pattern = p0 >= k;
    int lo, hi;
    if (text && pattern) { lo = -k; hi = k; }
    else if (text) { lo = k; hi = k; }
    else if (pattern) { lo = -k; hi = -k; }
    else { lo = 0; hi = 0; }
    int32_t* v = alloc(CM, s, lo, hi);
    if (retry) return wf_none();
    for (int kk = lo + lane; kk <= hi; kk += LW) v[kk - lo] = kOffsetNull;
    if (PB && pgb) bt_zero(v, 0, hi - lo);  // set_null_cell (:3454-3456)
    G::sync();
    if (lane == 0) {
      if (text) v[k - lo] = k;
      if (pattern) v[-k - lo] = 0;
    }
    if (PB && pgb) {
      G::sync();
      if (text) bt_init_cell(v, k - lo, 0, k);
      if (pattern) bt_init_cell(v, -k - lo, k, 0);
    }
    G::sync();
    WfD d;
    d.vals = v; d.lo = lo; d.hi = hi; d.a = lo; d.b = hi; d.flags = kPresent;
    d.adub = PB && pgb ? 0 : kAdUnknown;  // a fresh wavefront's occupancy is 0
    return d;
  }

  WFA_D void set_none(int s, int from_c, int to_c) {
    for (int c = from_c; c < to_c; ++c) put_ns(c, s, wf_none());
    G::sync();
  }
  WFA_D void set_m(int s, const WfD& d) {
    put_ns(CM, s, d);
    G::sync();
  }

  // ---- init_alignment, src/aligner.rs:846-1000 ------------------------------
  static WFA_D int gcd(int a, int b) {
    a = a < 0 ? -a : a;
    b = b < 0 ? -b : b;
    while (b) { int t = a % b; a = b; b = t; }
    return a;
  }
  WFA_D int score_step_gcd() const {
    int g;
    if (CLS == kEditClass) return 1;
    if (CLS == kLinearClass) g = gcd(P.mismatch, P.o1);
    else g = gcd(gcd(P.mismatch, P.o1 + P.e1), P.e1);
    if (TWO) g = gcd(gcd(g, P.o2 + P.e2), P.e2);
    if (ef() && P.match != 0 && (p0 > 0 || t0 > 0)) g = gcd(g, -P.match);
    return g < 1 ? 1 : g;
  }
  WFA_D void init_alignment() {
    cscore = 0;
    cidx = 0;
    gstep = score_step_gcd();
    gphase = 0;
    gshift = 0;
    dscope = scope;
    if (compact) {
      compact_depths();
      gshift = score_shift(gstep);
      dscope = ((scope - 1) >> gshift) + 1;
      if (P.desc_depth && dscope > P.desc_depth) retry = true;
      if (retry) return;
    }
    for (int i = lane; i < dscope * NC; i += LW) ws.ring[i] = wf_none();
    G::sync();
    hist_lo = -(n + scope + 2);
    hist_hi = m + scope + 2;
    num_null_steps = 0;
    status = WFA_STATUS_OK;
    end_score = -1; end_k = kDiagNull; end_off = kOffsetNull;
    hs.steps_wait = (hk() == WFA_HEURISTIC_WFADAPTIVE || hk() == WFA_HEURISTIC_BANDED_ADAPTIVE) ? hp2
                    : (hk() == WFA_HEURISTIC_XDROP || hk() == WFA_HEURISTIC_ZDROP) ? hp1 : 0;
    hs.max_sw_score = 0; hs.max_wf_score = 0; hs.max_sw_k = kDiagNull;
    hs.max_sw_off = kOffsetNull; hs.zdrop_last = 0;
    // Corrected mode (src/aligner.rs:912-947): no candidate yet; dominance
    // pruning only with begin-free seeds (at most 4 bases unless gap-linear)
    // and no heuristic that reads the wavefronts.
    corr = GEN && ef() && P.compat == WFA_COMPAT_CORRECTED && P.match < 0;
    c_has = false;
    const int bfree = imax(p0, t0);
    dom_on = GEN && corr && bfree > 0 && (CLS == kLinearClass || bfree <= 4) &&
             (hk() == WFA_HEURISTIC_NONE || hk() == WFA_HEURISTIC_BANDED_STATIC);
    if (dom_on) {
      dom_len = hist_hi - hist_lo + 1;
      if (!ws.dom || (int64_t)NC * dom_len > P.dom_words) { retry = true; return; }
      for (int64_t i = lane; i < (int64_t)NC * dom_len; i += LW) ws.dom[i] = -1;
      G::sync();
    }
    int lo0 = 0, hi0 = 0;
    bool seeds = ef() && P.match == 0;
    if (seeds) { lo0 = -p0; hi0 = t0; }
    int32_t* v = alloc(CM, 0, lo0, hi0);
    if (retry) return;
    for (int k = lo0 + lane; k <= hi0; k += LW) {
      int32_t val = k == 0 ? 0 : (k > 0 ? k : 0);  // seeds: (h,0) on k=h, (0,v) on k=-v
      v[k - lo0] = val;
    }
    if (PB && pgb) {
      // Chains start at (0, 0), then at the text seeds (0, h), then at the
      // pattern seeds (v, 0) (src/aligner.rs:962-992), numbered in that order.
      bt_used = 0;
      bi_used = 0;
      const int cnt = 1 + (seeds ? t0 + p0 : 0);
      if (cnt > P.bt_cap || cnt > P.bt_init_cap) { retry = true; return; }
      for (int i = lane; i < cnt; i += LW) {
        const int k = i == 0 ? 0 : i <= t0 ? i : -(i - t0);
        ws.btinit[i] = int2{k < 0 ? -k : 0, k > 0 ? k : 0};
        ws.bt[i] = uint2{(uint32_t)i, kBtNull};
        pcs(v)[k - lo0] = 0;
        pvs(v)[k - lo0] = (uint32_t)i;
      }
      bt_used = cnt;
      bi_used = cnt;
      cand_pc = 0; cand_pv = kBtNull; zd_pc = 0; zd_pv = kBtNull;
    }
    G::sync();
    WfD d;
    d.vals = v; d.lo = lo0; d.hi = hi0; d.a = lo0; d.b = hi0; d.flags = kPresent;
    d.adub = PB && pgb ? 0 : kAdUnknown;
    set_m(0, d);
  }

  // ---- med/low: compaction of the backtrace buffer ----------------------------
  // compact_bt_buffer (src/components.rs:231-279): keep the blocks reachable
  // from the live cells (offset >= 0) of the wavefronts still to be read and
  // from the kept chains (the Corrected candidate and the Z-drop best), move
  // them down in order, and translate the block indices of those cells and
  // chains.  The wavefronts still to be read are M of the last dm scores
  // that can hold one and I/D of the last d1 (d2), which own distinct cell
  // slots of the compact ring (the reference walks every wavefront of the
  // scope; the ones it adds are never read again).  The cells are those of
  // the initialised range, which later kernels read: the reference walks the
  // limits only, and a heuristic that narrows the limits leaves readable
  // cells outside them whose chains it would lose.  So compaction never
  // changes a result here.  ws.btmark: the mark bitmap, then the marked
  // blocks before each of its words.
  WFA_D void mark_chain(uint32_t idx) {
    int32_t guard = 0;
    while (idx != kBtNull && idx < (uint32_t)bt_used && guard++ <= bt_used) {
      const uint32_t bit = 1u << (idx & 31);
      if (G::atomic_or(&ws.btmark[idx >> 5], bit) & bit) return;
      idx = ws.bt[idx].y;
    }
  }
  WFA_D uint32_t moved_index(uint32_t idx, int nw) const {
    return ws.btmark[nw + (idx >> 5)] + (uint32_t)Warp::popc(ws.btmark[idx >> 5] & ((1u << (idx & 31)) - 1u));
  }
  // The cells of component c at score t (a multiple of the score step back
  // from the current one) whose chains compaction keeps; apply(pv) per cell.
  template <class F>
  WFA_D void live_cells(int c, int t, F&& apply) {
    if (t < 0) return;
    const WfD d = slot(c, t);
    if (!wf_present(d) || d.a > d.b) return;
    for (int k = d.a + lane; k <= d.b; k += LW)
      if (d.vals[k - d.a] >= 0) apply(pvs(d.vals)[k - d.a]);
  }
  template <class F>
  WFA_D void each_live_cell(F&& apply) {
    const int base = cscore - gphase;  // the last score that can hold a wavefront
    for (int j = 0; j < dm; ++j) live_cells(CM, base - j * gstep, apply);
    if (AFF)
      for (int j = 0; j < d1; ++j) {
        live_cells(CI1, base - j * gstep, apply);
        live_cells(CD1, base - j * gstep, apply);
      }
    if (TWO)
      for (int j = 0; j < d2; ++j) {
        live_cells(CI2, base - j * gstep, apply);
        live_cells(CD2, base - j * gstep, apply);
      }
  }
  WFA_D void compact_bt() {
    const int nw = (bt_used + 31) >> 5;
    for (int w = lane; w < nw; w += LW) ws.btmark[w] = 0;
    G::sync();
    each_live_cell([&](uint32_t& pv) { mark_chain(pv); });
    if (lane == 0) {
      if (c_has) mark_chain(cand_pv);
      mark_chain(zd_pv);
    }
    G::sync();
    if (lane == 0) {
      uint32_t run = 0;
      for (int w = 0; w < nw; ++w) {
        ws.btmark[nw + w] = run;
        run += (uint32_t)Warp::popc(ws.btmark[w]);
      }
    }
    G::sync();
    int32_t kept = 0;
    for (int i0 = 0; i0 < bt_used; i0 += LW) {
      const int i = i0 + lane;
      const bool mk = i < bt_used && (ws.btmark[i >> 5] >> (i & 31) & 1u);
      uint2 blk = uint2{0, 0};
      uint32_t to = 0;
      if (mk) {
        blk = ws.bt[i];
        if (blk.y != kBtNull) blk.y = moved_index(blk.y, nw);
        to = moved_index((uint32_t)i, nw);
      }
      int total;
      G::rank(mk, &total);  // every lane has read its block before any is written
      if (mk) ws.bt[to] = blk;
      kept += total;
      G::sync();
    }
    each_live_cell([&](uint32_t& pv) { if (pv != kBtNull) pv = moved_index(pv, nw); });
    // The kept chains are warp-uniform state: every lane translates them.
    if (c_has && cand_pv != kBtNull) cand_pv = moved_index(cand_pv, nw);
    if (zd_pv != kBtNull) zd_pv = moved_index(zd_pv, nw);
    G::sync();
    bt_used = kept;
  }

  // ---- med/low: the piggyback kernels' cells (src/compute/piggyback.rs) ------
  // Each cell copies (pcigar, prev) from the input its kernel picks and pushes
  // the operation taken.  Edit/linear (edit_kernel, :194-228): misms over del
  // over ins on ties; indel (:249-273): del over ins.  wi: insertion input
  // (cell k - 1), wx: mismatch input (cell k), wd: deletion input (cell k + 1).
  WFA_D void pb_edit_cell(const WfD& wi, const WfD& wx, const WfD& wd, int32_t* out, int L, int k,
                          bool indel) {
    const int32_t ins = rd(wi, k - 1) + 1, del = rd(wd, k + 1);
    uint32_t c, v;
    if (indel) {
      const bool d = imax(del, ins) == del;
      c = d ? pc_push(rpc(wd, k + 1), kPcDel) : pc_push(rpc(wi, k - 1), kPcIns);
      v = d ? rpv(wd, k + 1) : rpv(wi, k - 1);
    } else {
      const int32_t misms = rd(wx, k) + 1;
      const int32_t mx = imax(del, imax(ins, misms));
      const bool d = mx == del, x = mx == misms;
      c = x ? pc_push(rpc(wx, k), kPcMisms) : d ? pc_push(rpc(wd, k + 1), kPcDel) : pc_push(rpc(wi, k - 1), kPcIns);
      v = x ? rpv(wx, k) : d ? rpv(wd, k + 1) : rpv(wi, k - 1);
    }
    pcs(out)[k - L] = c;
    pvs(out)[k - L] = v;
  }
  // A gap cell (`gap`, :146-170): the extension on a tie with the M opening.
  struct PbGap {
    int32_t off;
    uint32_t c, v;
  };
  WFA_D PbGap pb_gap(const WfD& open, const WfD& ext, int kk, uint32_t op, int add) const {
    const int32_t o = rd(open, kk), e = rd(ext, kk);
    const bool x = e >= o;
    return PbGap{(x ? e : o) + add, pc_push(x ? rpc(ext, kk) : rpc(open, kk), op), x ? rpv(ext, kk) : rpv(open, kk)};
  }
  // Affine / two-piece affine (affine_kernel :364-392, affine2p_kernel
  // :483-527): I and D from their gaps; M takes misms, else D2, D1, I2, I1
  // (later checks win ties) and pushes an X (the gap close) on the chain.
  WFA_D void pb_affine_cell(const WfD& mm, const WfD& mo1, const WfD& i1e, const WfD& d1e, const WfD& mo2,
                            const WfD& i2e, const WfD& d2e, bool two, int32_t* om, int L, int32_t* oi1,
                            int32_t* od1, int32_t* oi2, int32_t* od2, int lo, int k) {
    const PbGap i1 = pb_gap(mo1, i1e, k - 1, kPcIns, 1), d1 = pb_gap(mo1, d1e, k + 1, kPcDel, 0);
    pcs(oi1)[k - lo] = i1.c; pvs(oi1)[k - lo] = i1.v;
    pcs(od1)[k - lo] = d1.c; pvs(od1)[k - lo] = d1.v;
    const int32_t misms = rd(mm, k) + 1;
    int32_t mx;
    uint32_t c, v;
    if (!two) {
      mx = imax(d1.off, imax(misms, i1.off));
      const bool d = mx == d1.off;
      c = d ? d1.c : i1.c;
      v = d ? d1.v : i1.v;
    } else {
      const PbGap i2 = pb_gap(mo2, i2e, k - 1, kPcIns, 1), d2 = pb_gap(mo2, d2e, k + 1, kPcDel, 0);
      pcs(oi2)[k - lo] = i2.c; pvs(oi2)[k - lo] = i2.v;
      pcs(od2)[k - lo] = d2.c; pvs(od2)[k - lo] = d2.v;
      mx = imax(imax(imax(i1.off, i2.off), imax(d1.off, d2.off)), misms);
      const bool s2 = mx == i2.off, t1 = mx == d1.off, t2 = mx == d2.off;
      c = t2 ? d2.c : t1 ? d1.c : s2 ? i2.c : i1.c;
      v = t2 ? d2.v : t1 ? d1.v : s2 ? i2.v : i1.v;
    }
    const bool x = mx == misms;
    pcs(om)[k - L] = pc_push(x ? rpc(mm, k) : c, kPcMisms);
    pvs(om)[k - L] = x ? rpv(mm, k) : v;
  }

  // ---- compute steps ----------------------------------------------------------
  // compute_edit_step, src/aligner.rs:1769-1864
  WFA_D void compute_edit(int s) {
    WfD prev = get(CM, s - 1);
    if (wf_is_null(prev)) { ++num_null_steps; set_m(s, wf_none()); return; }
    num_null_steps = 0;
    int lo = imax(prev.lo - 1, hist_lo + 1), hi = imin(prev.hi + 1, hist_hi - 1);
    if (lo > hi) { set_m(s, wf_none()); return; }
    // NULL the cells the kernel reads beyond prev's limits (inside its
    // initialised range only; outside it they already read as NULL).
    if (lane == 0) {
      int ks[4] = {prev.lo - 2, prev.lo - 1, prev.hi + 1, prev.hi + 2};
      int4 hr = modular || (PB && pgb) ? int4{0, -1, 0, 0} : ws.hist[(int64_t)(s - 1) * hist_nc];
      for (int i = 0; i < 4; ++i) {
        if (ks[i] >= prev.a && ks[i] <= prev.b) {
          prev.vals[ks[i] - prev.a] = kOffsetNull;
          if (PB && pgb) { pcs(prev.vals)[ks[i] - prev.a] = 0; pvs(prev.vals)[ks[i] - prev.a] = 0; }
        }
        if (hr.w && ks[i] >= hr.x && ks[i] <= hr.y) ws.harena[hr.z + ks[i] - hr.x] = kOffsetNull;
      }
    }
    G::sync();
    int32_t* out = alloc(CM, s, lo, hi);
    if (retry) return;
    bool indel = P.metric == WFA_METRIC_INDEL;
    int vmin = INT_MAX, vmax = INT_MIN;
    for (int k = lo + lane; k <= hi; k += LW) {
      int32_t ins = rd(prev, k - 1), del = rd(prev, k + 1), mx;
      if (indel) mx = imax(del, ins + 1);
      else mx = imax(del, imax(ins, rd(prev, k)) + 1);
      if (PB && pgb) pb_edit_cell(prev, prev, prev, out, lo, k, indel);
      if (!cell_in_bounds(mx, k, n, m)) mx = kOffsetNull;
      out[k - lo] = mx;
      if (mx != kOffsetNull) { vmin = imin(vmin, k); vmax = imax(vmax, k); }
    }
    // C offloads edit/indel every PCIGAR_MAX_LENGTH scores (src/aligner.rs:1848-1852).
    if (PB && pgb && s % kPcMaxLength == 0) {
      G::sync();
      offload_linear_cells(out, lo, lo, hi);
      if (retry) return;
    }
    vmin = G::min(vmin);
    vmax = G::max(vmax);
    set_m(s, finish(out, lo, lo, hi, vmin, vmax));
  }

  // compute_linear_step, src/aligner.rs:1867-2003
  WFA_D void compute_linear(int s) {
    WfD mi = get(CM, s - P.mismatch), gp = get(CM, s - P.o1);
    int bk;
    if (wf_is_null(mi) && wf_is_null(gp)) {
      ++num_null_steps;
      WfD d = wf_none();
      if (begin_k(s, bk)) d = endsfree_null_m(s, bk);
      set_m(s, d);
      return;
    }
    num_null_steps = 0;
    if (wf_is_null(mi)) mi = wf_none();
    if (wf_is_null(gp)) gp = wf_none();
    int lo = imin(mi.lo, gp.lo - 1), hi = imax(mi.hi, gp.hi + 1);
    clamp_band(lo, hi);
    lo = imax(lo, hist_lo + 1);
    hi = imin(hi, hist_hi - 1);
    if (lo > hi) { set_m(s, wf_none()); return; }
    bool bf = begin_k(s, bk);
    int L = bf ? imin(lo, -bk) : lo, H = bf ? imax(hi, bk) : hi;
    int32_t* out = alloc(CM, s, L, H);
    if (retry) return;
    int32_t lin_occ = 0;
    int vmin = INT_MAX, vmax = INT_MIN;
    for (int k = lo + lane; k <= hi; k += LW) {
      int32_t a = rd(mi, k) + 1, ins = rd(gp, k - 1) + 1, del = rd(gp, k + 1);
      int32_t mx = imax(del, imax(ins, a));
      if (PB && pgb) pb_edit_cell(gp, mi, gp, out, L, k, false);
      if (!cell_in_bounds(mx, k, n, m)) mx = kOffsetNull;
      out[k - L] = mx;
      if (mx != kOffsetNull) { vmin = imin(vmin, k); vmax = imax(vmax, k); }
    }
    if (PB && pgb) {  // offload_linear (src/compute/piggyback.rs:590-607)
      G::sync();
      lin_occ = imax(occ_of(gp), occ_of(mi)) + 1;
      if (lin_occ >= kPcMaxLength) lin_occ = offload_linear_cells(out, L, lo, hi);
      if (retry) return;
    }
    WfD r;
    if (bf) {
      endsfree_init(out, L, lo, hi, bk);
      r = trim_pass(out, L, lo, hi);
    } else {
      vmin = G::min(vmin);
      vmax = G::max(vmax);
      r = finish(out, L, lo, hi, vmin, vmax);
    }
    if (PB && pgb) r.adub = lin_occ;
    set_m(s, r);
  }

  // compute_affine_step (src/aligner.rs:2006-2193) and compute_affine2p_step
  // (:2201-2553); the recurrences of src/compute/affine.rs:318-351 and
  // src/compute/affine2p.rs:208-233.
  WFA_D void compute_affine(int s) {
    const int x = P.mismatch, oe1 = P.o1 + P.e1, e1 = P.e1;
    const int oe2 = TWO ? P.o2 + P.e2 : 0, e2 = TWO ? P.e2 : 0;
    int bk;
    // Null step (every input missing or empty), decided on the flags alone.
    bool any_live = live(CM, s - x) || live(CM, s - oe1) || live(CI1, s - e1) || live(CD1, s - e1);
    if (TWO) any_live = any_live || live(CM, s - oe2) || live(CI2, s - e2) || live(CD2, s - e2);
    if (!any_live) {
      ++num_null_steps;
      for (int c = 1; c < NC; ++c) put_ns(c, s, wf_none());
      WfD d = wf_none();
      if (begin_k(s, bk)) d = endsfree_null_m(s, bk);
      set_m(s, d);
      return;
    }
    WfD mm = get(CM, s - x), mo1 = get(CM, s - oe1);
    WfD i1e = get(CI1, s - e1), d1e = get(CD1, s - e1);
    WfD mo2 = wf_none(), i2e = wf_none(), d2e = wf_none();
    if (TWO) { mo2 = get(CM, s - oe2); i2e = get(CI2, s - e2); d2e = get(CD2, s - e2); }
    num_null_steps = 0;
    if (wf_is_null(mm)) mm = wf_none();
    if (wf_is_null(mo1)) mo1 = wf_none();
    if (wf_is_null(i1e)) i1e = wf_none();
    if (wf_is_null(d1e)) d1e = wf_none();
    if (TWO) {
      if (wf_is_null(mo2)) mo2 = wf_none();
      if (wf_is_null(i2e)) i2e = wf_none();
      if (wf_is_null(d2e)) d2e = wf_none();
    }
    bool affine_kernel = true;
    if (TWO) {
      bool i2a = wf_present(mo2) || wf_present(i2e), d2a = wf_present(mo2) || wf_present(d2e);
      affine_kernel = !i2a && !d2a;
    }
    // Range union; absent inputs contribute the null bounds (1, -1).
    int lo = imin(imin(mm.lo, mo1.lo - 1), imin(i1e.lo + 1, d1e.lo - 1));
    int hi = imax(imax(mm.hi, mo1.hi + 1), imax(i1e.hi + 1, d1e.hi - 1));
    if (TWO) {
      lo = imin(lo, imin(mo2.lo - 1, imin(i2e.lo + 1, d2e.lo - 1)));
      hi = imax(hi, imax(mo2.hi + 1, imax(i2e.hi + 1, d2e.hi - 1)));
    }
    clamp_band(lo, hi);
    if (lo <= hi) { lo = imax(lo, hist_lo + 1); hi = imin(hi, hist_hi - 1); }
    if (lo > hi) {
      for (int c = 1; c < NC; ++c) put_ns(c, s, wf_none());
      set_m(s, wf_none());
      return;
    }
    bool bf = begin_k(s, bk);
    int L = bf ? imin(lo, -bk) : lo, H = bf ? imax(hi, bk) : hi;
    int32_t* om = alloc(CM, s, L, H);
    int32_t* oi1 = alloc(CI1, s, lo, hi);
    int32_t* od1 = alloc(CD1, s, lo, hi);
    int32_t *oi2 = nullptr, *od2 = nullptr;
    if (TWO && !affine_kernel) { oi2 = alloc(CI2, s, lo, hi); od2 = alloc(CD2, s, lo, hi); }
    if (retry) return;
    if constexpr (UNR > 1) {
      if (!bf) {
        affine_wide(s, lo, hi, mm, mo1, i1e, d1e, mo2, i2e, d2e, TWO && !affine_kernel, om, oi1, od1,
                    oi2, od2);
        return;
      }
    }
    int mn_m = INT_MAX, mx_m = INT_MIN, mn_i1 = INT_MAX, mx_i1 = INT_MIN, mn_d1 = INT_MAX, mx_d1 = INT_MIN;
    int mn_i2 = INT_MAX, mx_i2 = INT_MIN, mn_d2 = INT_MAX, mx_d2 = INT_MIN;
    const bool two = TWO && !affine_kernel;
    for (int k0 = lo + lane; k0 <= hi; k0 += LW * UNR) {
      // Inputs of UNR diagonals first (reads stay inside each input's
      // initialised range, also for k > hi), then the results.
      int32_t vi1[UNR], vd1[UNR], vm[UNR], vi2[UNR], vd2[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int k = k0 + u * LW;
        vi1[u] = imax(rd(mo1, k - 1), rd(i1e, k - 1)) + 1;
        vd1[u] = imax(rd(mo1, k + 1), rd(d1e, k + 1));
        vm[u] = rd(mm, k) + 1;
        if (two) {
          vi2[u] = imax(rd(mo2, k - 1), rd(i2e, k - 1)) + 1;
          vd2[u] = imax(rd(mo2, k + 1), rd(d2e, k + 1));
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int k = k0 + u * LW;
        if (k > hi) break;
        const int32_t i1 = vi1[u], d1 = vd1[u];
        int32_t mx;
        if (!two) {
          mx = imax(vm[u], imax(i1, d1));
        } else {
          const int32_t i2 = vi2[u], d2 = vd2[u];
          mx = imax(vm[u], imax(imax(i1, i2), imax(d1, d2)));
          oi2[k - lo] = i2;
          od2[k - lo] = d2;
          if (cell_in_bounds(i2, k, n, m)) { mn_i2 = imin(mn_i2, k); mx_i2 = imax(mx_i2, k); }
          if (cell_in_bounds(d2, k, n, m)) { mn_d2 = imin(mn_d2, k); mx_d2 = imax(mx_d2, k); }
        }
        if (PB && pgb)
          pb_affine_cell(mm, mo1, i1e, d1e, mo2, i2e, d2e, two, om, L, oi1, od1, oi2, od2, lo, k);
        if (!cell_in_bounds(mx, k, n, m)) mx = kOffsetNull;
        om[k - L] = mx;
        oi1[k - lo] = i1;
        od1[k - lo] = d1;
        if (mx != kOffsetNull) { mn_m = imin(mn_m, k); mx_m = imax(mx_m, k); }
        if (cell_in_bounds(i1, k, n, m)) { mn_i1 = imin(mn_i1, k); mx_i1 = imax(mx_i1, k); }
        if (cell_in_bounds(d1, k, n, m)) { mn_d1 = imin(mn_d1, k); mx_d1 = imax(mx_d1, k); }
      }
    }
    // Med/low: occupancies and offload (offload_affine / offload_affine2p,
    // src/compute/piggyback.rs:635-705), before the trims as the reference.
    int32_t o_m = 0, o_i1 = 0, o_d1 = 0, o_i2 = 0, o_d2 = 0;
    if (PB && pgb) {
      G::sync();
      o_i1 = occ_gap(mo1, i1e);
      o_d1 = occ_gap(mo1, d1e);
      o_m = imax(occ_of(mm), imax(o_i1, o_d1));
      if (two) {
        o_i2 = occ_gap(mo2, i2e);
        o_d2 = occ_gap(mo2, d2e);
        o_m = imax(o_m, imax(o_i2, o_d2));
      }
      o_m = offload_component(om, L, lo, hi, o_m + 1);
      o_i1 = offload_component(oi1, lo, lo, hi, o_i1);
      o_d1 = offload_component(od1, lo, lo, hi, o_d1);
      if (two) {
        o_i2 = offload_component(oi2, lo, lo, hi, o_i2);
        o_d2 = offload_component(od2, lo, lo, hi, o_d2);
      }
      if (retry) return;
    }
    mn_i1 = G::min(mn_i1); mx_i1 = G::max(mx_i1);
    mn_d1 = G::min(mn_d1); mx_d1 = G::max(mx_d1);
    WfD r = finish(oi1, lo, lo, hi, mn_i1, mx_i1);
    if (PB && pgb) r.adub = o_i1;
    put_ns(CI1, s, r);
    r = finish(od1, lo, lo, hi, mn_d1, mx_d1);
    if (PB && pgb) r.adub = o_d1;
    put_ns(CD1, s, r);
    if (TWO) {
      if (affine_kernel) {
        put_ns(CI2, s, wf_none());
        put_ns(CD2, s, wf_none());
      } else {
        mn_i2 = G::min(mn_i2); mx_i2 = G::max(mx_i2);
        mn_d2 = G::min(mn_d2); mx_d2 = G::max(mx_d2);
        r = finish(oi2, lo, lo, hi, mn_i2, mx_i2);
        if (PB && pgb) r.adub = o_i2;
        put_ns(CI2, s, r);
        r = finish(od2, lo, lo, hi, mn_d2, mx_d2);
        if (PB && pgb) r.adub = o_d2;
        put_ns(CD2, s, r);
      }
    }
    if (bf) {
      int mlo = lo, mhi = hi;
      endsfree_init(om, L, mlo, mhi, bk);
      r = trim_pass(om, L, mlo, mhi);
    } else {
      mn_m = G::min(mn_m); mx_m = G::max(mx_m);
      r = finish(om, L, lo, hi, mn_m, mx_m);
    }
    if (PB && pgb) r.adub = o_m;
    set_m(s, r);
  }


  // ---- wide affine compute (UNR > 1: BiWFA) -----------------------------------
  // The same cells as compute_affine's loop.  Cells whose every input lies
  // inside the input's initialised range are read without range checks, UNR
  // per lane per pass; the trim (trim_ends, src/compute/mod.rs:14-49) is
  // found by scanning in from both ends of each stored row.
  template <bool CHK, int U>
  WFA_D void wide_pass(int kb, int ke, int lo, const WfD& mm, const WfD& mo1, const WfD& i1e,
                       const WfD& d1e, const WfD& mo2, const WfD& i2e, const WfD& d2e, bool two,
                       int32_t* om, int32_t* oi1, int32_t* od1, int32_t* oi2, int32_t* od2) {
    for (int k0 = kb + lane; k0 <= ke; k0 += LW * U) {
      int32_t vi1[U], vd1[U], vm[U], vi2[U], vd2[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = imin(k0 + u * LW, ke);  // lanes past ke repeat ke's reads
        if (CHK) {
          vi1[u] = imax(rd(mo1, k - 1), rd(i1e, k - 1)) + 1;
          vd1[u] = imax(rd(mo1, k + 1), rd(d1e, k + 1));
          vm[u] = rd(mm, k) + 1;
          if (two) {
            vi2[u] = imax(rd(mo2, k - 1), rd(i2e, k - 1)) + 1;
            vd2[u] = imax(rd(mo2, k + 1), rd(d2e, k + 1));
          }
        } else {
          vi1[u] = imax(mo1.vals[k - 1 - mo1.a], i1e.vals[k - 1 - i1e.a]) + 1;
          vd1[u] = imax(mo1.vals[k + 1 - mo1.a], d1e.vals[k + 1 - d1e.a]);
          vm[u] = mm.vals[k - mm.a] + 1;
          if (two) {
            vi2[u] = imax(mo2.vals[k - 1 - mo2.a], i2e.vals[k - 1 - i2e.a]) + 1;
            vd2[u] = imax(mo2.vals[k + 1 - mo2.a], d2e.vals[k + 1 - d2e.a]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * LW;
        if (k > ke) break;
        int32_t mx = imax(vm[u], imax(vi1[u], vd1[u]));
        if (two) mx = imax(mx, imax(vi2[u], vd2[u]));
        if (!cell_in_bounds(mx, k, n, m)) mx = kOffsetNull;
        om[k - lo] = mx;
        oi1[k - lo] = vi1[u];
        od1[k - lo] = vd1[u];
        if (two) {
          oi2[k - lo] = vi2[u];
          od2[k - lo] = vd2[u];
        }
      }
    }
  }
  // Highest / lowest k of row[lo..hi] (row[0] is cell lo) holding an
  // in-bounds offset; INT_MIN / INT_MAX if none.
  WFA_D int row_last(const int32_t* row, int lo, int hi) const {
    for (int top = hi; top >= lo; top -= LW) {
      const int k = top - lane;
      const bool ok = k >= lo && cell_in_bounds(row[k - lo], k, n, m);
      const int best = G::max(ok ? k : INT_MIN);
      if (best != INT_MIN) return best;
    }
    return INT_MIN;
  }
  WFA_D int row_first(const int32_t* row, int lo, int hi) const {
    for (int bot = lo; bot <= hi; bot += LW) {
      const int k = bot + lane;
      const bool ok = k <= hi && cell_in_bounds(row[k - lo], k, n, m);
      const int best = G::min(ok ? k : INT_MAX);
      if (best != INT_MAX) return best;
    }
    return INT_MAX;
  }
  WFA_D void affine_wide(int s, int lo, int hi, const WfD& mm, const WfD& mo1, const WfD& i1e,
                         const WfD& d1e, const WfD& mo2, const WfD& i2e, const WfD& d2e, bool two,
                         int32_t* om, int32_t* oi1, int32_t* od1, int32_t* oi2, int32_t* od2) {
    // Interior: every read of every input inside its initialised range
    // (mm at k, mo1/mo2 at k-1 and k+1, i1e/i2e at k-1, d1e/d2e at k+1).
    int ilo = imax(mm.a, imax(mo1.a + 1, imax(i1e.a + 1, d1e.a - 1)));
    int ihi = imin(mm.b, imin(mo1.b - 1, imin(i1e.b + 1, d1e.b - 1)));
    if (two) {
      ilo = imax(ilo, imax(mo2.a + 1, imax(i2e.a + 1, d2e.a - 1)));
      ihi = imin(ihi, imin(mo2.b - 1, imin(i2e.b + 1, d2e.b - 1)));
    }
    ilo = imax(ilo, lo);
    ihi = imin(ihi, hi);
    if (ilo > ihi) { ilo = hi + 1; ihi = hi; }  // no interior: all checked
    // Edges (checked, one diagonal per lane per pass), then the interior.
    for (int e = 0; e < 2; ++e) {
      const int kb = e == 0 ? lo : ihi + 1, ke = e == 0 ? ilo - 1 : hi;
      if (kb <= ke)
        wide_pass<true, 1>(kb, ke, lo, mm, mo1, i1e, d1e, mo2, i2e, d2e, two, om, oi1, od1, oi2, od2);
    }
    if (ilo <= ihi)
      wide_pass<false, UNR>(ilo, ihi, lo, mm, mo1, i1e, d1e, mo2, i2e, d2e, two, om, oi1, od1, oi2, od2);
    G::sync();  // the scans read cells other lanes stored
    // Trims of the rows I1, D1 (, I2, D2) and M: the top and then the bottom
    // LW cells of every row are checked together; a row whose end
    // chunk holds no in-bounds cell continues with a scan.
    constexpr int RN = TWO ? 5 : 3;
    int32_t* rows[RN];
    rows[0] = oi1;
    rows[1] = od1;
    if (TWO) { rows[2] = oi2; rows[3] = od2; }
    rows[RN - 1] = om;
    int last[RN], first[RN];
    {
      const int k = hi - lane;
      int32_t v[RN];
#pragma unroll
      for (int r = 0; r < RN; ++r) v[r] = (k >= lo && (two || r < 2 || r == RN - 1)) ? rows[r][k - lo] : kOffsetNull;
#pragma unroll
      for (int r = 0; r < RN; ++r) last[r] = G::max(cell_in_bounds(v[r], k, n, m) ? k : INT_MIN);
    }
#pragma unroll
    for (int r = 0; r < RN; ++r)
      if (last[r] == INT_MIN && (two || r < 2 || r == RN - 1) && hi - LW >= lo)
        last[r] = row_last(rows[r], lo, hi - LW);
    {
      const int k = lo + lane;
      int32_t v[RN];
#pragma unroll
      for (int r = 0; r < RN; ++r) v[r] = (k <= last[r]) ? rows[r][k - lo] : kOffsetNull;
#pragma unroll
      for (int r = 0; r < RN; ++r) first[r] = G::min(cell_in_bounds(v[r], k, n, m) ? k : INT_MAX);
    }
#pragma unroll
    for (int r = 0; r < RN; ++r)
      if (first[r] == INT_MAX && last[r] != INT_MIN)
        first[r] = row_first(rows[r] + LW, lo + LW, last[r]);
    // Antidiagonal bounds: I[k] = max(M'[k-1], I'[k-1]) + 1 and
    // D[k] = max(M'[k+1], D'[k+1]) both lie one antidiagonal above a source
    // cell.  M's bound is set by the extend step.
    WfD r;
    r = finish(oi1, lo, lo, hi, first[0], last[0]); r.adub = imax(ad_of(mo1), ad_of(i1e)) + 1; put_ns(CI1, s, r);
    r = finish(od1, lo, lo, hi, first[1], last[1]); r.adub = imax(ad_of(mo1), ad_of(d1e)) + 1; put_ns(CD1, s, r);
    if (TWO) {
      if (two) {
        r = finish(oi2, lo, lo, hi, first[2], last[2]); r.adub = imax(ad_of(mo2), ad_of(i2e)) + 1; put_ns(CI2, s, r);
        r = finish(od2, lo, lo, hi, first[3], last[3]); r.adub = imax(ad_of(mo2), ad_of(d2e)) + 1; put_ns(CD2, s, r);
      } else {
        put_ns(CI2, s, wf_none());
        put_ns(CD2, s, wf_none());
      }
    }
    set_m(s, finish(om, lo, lo, hi, first[RN - 1], last[RN - 1]));
  }

  WFA_D void compute_step(int s) {
    if (PB && pgb) mbase = nullptr;  // set again if this score allocates an M
    if (CLS == kEditClass) compute_edit(s);
    else if (CLS == kLinearClass) compute_linear(s);
    else compute_affine(s);
    // Dominance pruning of the outputs, after their trims (src/aligner.rs:
    // 1999-2001, 2187-2191, 2541-2550): M without recording, the gap
    // components recording the offsets they keep.
    if (GEN && dom_on && !retry)
      for (int c = 0; c < NC; ++c) dom_prune(s, c, c != CM);
  }

  // ---- Compat::Corrected ends-free ---------------------------------------------
  // NULL cells [from, to] of a stored wavefront (inside its initialised range).
  WFA_D void null_cells(const WfD& d, int from, int to) {
    from = imax(from, d.a);
    to = imin(to, d.b);
    for (int k = from + lane; k <= to; k += LW) d.vals[k - d.a] = kOffsetNull;
  }
  // Wavefront::trim_nulled (src/wavefront.rs:463-490) of component c at s.
  WFA_D void trim_nulled(int c, int s, int lo, int hi) {
    WfD d = slot(c, s);
    G::sync();
    if (!wf_present(d) || (d.flags & kNullFlag) || d.lo > d.hi || (lo <= d.lo && hi >= d.hi)) return;
    const int nlo = imax(lo, d.lo), nhi = imin(hi, d.hi);
    if (nlo > nhi) {
      null_cells(d, d.lo, d.hi);
      d.flags |= kNullFlag;
    } else {
      null_cells(d, d.lo, nlo - 1);
      null_cells(d, nhi + 1, d.hi);
    }
    d.lo = nlo;
    d.hi = nhi;
    put(c, s, d);
  }
  // endsfree_prune (src/aligner.rs:1214-1255): null, in every component at
  // s, the diagonals farther than (total - s) / -match from the end diagonal.
  WFA_D void ef_prune(int s, int total) {
    const int radius = (total - s) / -P.match, kend = m - n;
    for (int c = 0; c < NC; ++c) trim_nulled(c, s, kend - radius, kend + radius);
  }
  // endsfree_dominance_prune (src/aligner.rs:1257-1320): trim from the ends
  // the cells of component c at s that reach no further than a cell of c did
  // at an earlier score; with `record`, keep the kept offsets.
  WFA_D void dom_prune(int s, int c, bool record) {
    WfD d = slot(c, s);
    G::sync();
    if (!wf_present(d) || d.lo > d.hi) return;
    int32_t* b = ws.dom + (int64_t)c * dom_len + (d.lo - hist_lo);
    const int cnt = d.hi - d.lo + 1;
    WFA_CHECK(d.lo >= hist_lo && d.hi - hist_lo < dom_len, return);
    int first = cnt, last = -1;
    for (int i = lane; i < cnt; i += LW)
      if (d.vals[d.lo + i - d.a] > b[i]) { first = imin(first, i); last = imax(last, i); }
    first = G::min(first);
    last = G::max(last) + 1;  // one past the last kept cell
    if (first >= cnt) last = first;
    if (record)
      for (int i = first + lane; i < last; i += LW) b[i] = imax(b[i], d.vals[d.lo + i - d.a]);
    null_cells(d, d.lo, d.lo + first - 1);
    null_cells(d, d.lo + last, d.hi);
    if (first == last) {
      d.lo = 1;
      d.hi = 0;
      d.flags |= kNullFlag;
    } else {
      d.hi = d.lo + last - 1;
      d.lo = d.lo + first;
    }
    G::sync();
    put(c, s, d);
  }
  // endsfree_dominance_update (src/aligner.rs:1322-1338): M after extend.
  WFA_D void dom_update(int s) {
    WfD d = slot(CM, s);
    if (wf_is_null(d) || d.lo > d.hi) return;
    int32_t* b = ws.dom + (d.lo - hist_lo);
    WFA_CHECK(d.lo >= hist_lo && d.hi - hist_lo < dom_len, return);
    for (int k = d.lo + lane; k <= d.hi; k += LW) b[k - d.lo] = imax(b[k - d.lo], d.vals[k - d.a]);
    G::sync();
  }
  // extend_matches_packed_endsfree_best (src/extend.rs:179-232): extend every
  // cell and find the free-end cell leaving the fewest bases to its free end
  // gap (endsfree_left, src/termination.rs:65-86), the lowest diagonal on ties.
  WFA_D bool extend_best(WfD& d, int& rk, int& roff, int& rleft) {
    int bl = INT_MAX, bkk = INT_MAX;
    for (int k = d.lo + lane; k <= d.hi; k += LW) {
      int32_t off = d.vals[k - d.a];
      if (off < 0) continue;  // NULL (M offsets are valid or NULL)
      int v = off - k, h = off;
      int R = imin(n - v, m - h);
      if (R > 0) {
        off += lcp_fwd(pat, v, txt, h, R);
        d.vals[k - d.a] = off;
        v = off - k;
        h = off;
      }
      const bool by_t = h >= m && n - v <= pf, by_p = v >= n && m - h <= tf;
      if (by_t || by_p) {
        const int left = by_t && by_p ? imin(n - v, m - h) : by_t ? n - v : m - h;
        if (left < bl) { bl = left; bkk = k; }
      }
    }
    G::sync();
    rleft = G::min(bl);
    if (rleft == INT_MAX) return false;
    rk = G::min(bl == rleft ? bkk : INT_MAX);
    roff = d.vals[rk - d.a];
    return true;
  }
  // extend_endsfree_corrected (src/aligner.rs:1123-1211).
  WFA_D bool extend_step_corrected(int score) {
    const bool prune = hk() == WFA_HEURISTIC_NONE || hk() == WFA_HEURISTIC_BANDED_STATIC;
    if (prune && c_has && c_total > score) ef_prune(score, c_total);
    WfD d = slot(CM, score);
    G::sync();
    if (wf_present(d)) {
      int k, off, left;
      if (extend_best(d, k, off, left)) {
        const int total = score + (-P.match) * left;
        if (!c_has || total < c_total) {
          c_has = true; c_total = total; c_score = score; c_k = k; c_off = off;
          if (pgb) m_bt(k, cand_pc, cand_pv);  // the candidate's chain (src/aligner.rs:1155-1160)
          if (prune && total > score) ef_prune(score, total);
        }
      }
      if (dom_on) dom_update(score);
    }
    if (c_has && c_total <= score) {  // no later cell can beat the candidate
      end_score = c_score; end_k = c_k; end_off = c_off;
      status = WFA_STATUS_END_REACHED;
      return true;
    }
    bool done;
    if (!wf_present(d)) done = !c_has && num_null_steps > scope;
    else done = hk() != WFA_HEURISTIC_NONE && apply_heuristic(score);
    if (done) {
      if (c_has) {
        end_score = c_score; end_k = c_k; end_off = c_off;
        status = WFA_STATUS_END_REACHED;
      } else {
        status = WFA_STATUS_END_UNREACHABLE;
      }
      return true;
    }
    return false;
  }

  // ---- extend ----------------------------------------------------------------
  // extend_matches_packed_end2end (src/extend.rs:47-70): extend every
  // diagonal of [lo, hi] with offset >= 0.  Returns the lowest diagonal
  // meeting the ends-free termination (termination_endsfree,
  // src/termination.rs:31-58) when `endsfree_term`, else INT_MAX.
  WFA_D int extend_wf(WfD& d, bool endsfree_term, int& term_off) {
    int best = INT_MAX, best_off = 0;
    for (int k = d.lo + lane; k <= d.hi; k += LW) {
      int32_t off = d.vals[k - d.a];
      if (off >= 0) {
        int v = off - k, h = off;
        int R = imin(n - v, m - h);
        if (R > 0) {
          off += lcp_fwd(pat, v, txt, h, R);
          d.vals[k - d.a] = off;
        }
        if (endsfree_term && k < best) {
          int hh = off, vv = off - k;
          if ((hh >= m && n - vv <= pf) || (vv >= n && m - hh <= tf)) { best = k; best_off = off; }
        }
      }
    }
    G::sync();
    if (endsfree_term) {
      int kb = G::min(best);
      if (kb != INT_MAX) term_off = d.vals[kb - d.a];
      (void)best_off;
      return kb;
    }
    return INT_MAX;
  }

  // ---- heuristics: src/heuristic.rs:167-520, src/aligner.rs:1644-1766 ---------
  WFA_D int32_t dist(const WfD& d, int k) const {  // wf_distance_end2end
    int32_t off = d.vals[k - d.a];
    if (off < 0) return INT_MAX;
    return imax(n - (off - k), m - off);
  }
  // SW score of cell k (compute_sw_scores); `valid` false for offset < 0.
  WFA_D int32_t sw_score(const WfD& d, int k, int score, bool& valid) const {
    int32_t off = d.vals[k - d.a];
    valid = off >= 0;
    if (!valid) return 0;
    int swg = P.match != 0 ? -P.match : 1;
    bool bfree = P.match == 0 && ef();
    int fv = k < 0 ? imin(-k, bfree ? p0 : 0) : 0;
    int fh = k > 0 ? imin(k, bfree ? t0 : 0) : 0;
    int v = off - k - fv, h = off - fh;
    return (swg * (v + h) - score) / 2;
  }
  // Warp max of the SW scores with the lowest diagonal among the maxima.
  WFA_D void sw_max(const WfD& d, int score, int& cmax, int& ck, int& coff) {
    int best = INT_MIN, bk = INT_MAX;
    for (int k = d.lo + lane; k <= d.hi; k += LW) {
      bool ok;
      int sw = sw_score(d, k, score, ok);
      if (ok && (sw > best || (sw == best && k < bk))) { best = sw; bk = k; }
    }
    cmax = G::max(best);
    int cand = (best == cmax) ? bk : INT_MAX;
    ck = G::min(cand);
    if (cmax == INT_MIN) { ck = 0; coff = 0; }
    else coff = d.vals[ck - d.a];
  }

  // heuristic_cutoff; returns true on a Z-drop.  d is M at `score`.
  WFA_D bool heuristic_cutoff(WfD& d, int score) {
    if (d.lo > d.hi) return false;
    hs.steps_wait -= 1;
    switch (hk()) {
      case WFA_HEURISTIC_WFADAPTIVE: {
        if (hs.steps_wait > 0) return false;
        int blo = d.lo, bhi = d.hi;
        if (bhi - blo + 1 < hp0) return false;
        int mn = INT_MAX;
        for (int k = blo + lane; k <= bhi; k += LW) mn = imin(mn, dist(d, k));
        int min_d = imin(G::min(mn), imax(n, m));
        int ak = m - n, thr = hp1;
        auto ok = [&](int k) { return (int32_t)((uint32_t)dist(d, k) - (uint32_t)min_d) <= thr; };
        int top = imin(ak, d.hi), nlo = d.lo;
        if (top > d.lo) {
          int f = INT_MAX;
          for (int k = d.lo + lane; k < top; k += LW) if (ok(k)) { f = k; break; }
          f = G::min(f);
          nlo = imin(f, top);
        }
        int bottom = imax(ak, nlo), nhi = d.hi;
        if (d.hi > bottom) {
          int l = INT_MIN;
          for (int k = d.hi - lane; k > bottom; k -= LW) if (ok(k)) { l = k; break; }
          l = G::max(l);
          nhi = imax(l, bottom);
        }
        d.lo = nlo;
        d.hi = nhi;
        hs.steps_wait = hp2;
        return false;
      }
      case WFA_HEURISTIC_BANDED_STATIC:
        if (d.lo < hp0) d.lo = hp0;
        if (d.hi > hp1) d.hi = hp1;
        return false;
      case WFA_HEURISTIC_BANDED_ADAPTIVE: {
        if (hs.steps_wait > 0) return false;
        int lo = d.lo, hi = d.hi, len = hi - lo + 1;
        if (len < 4) return false;
        int maxlen = hp1 - hp0 + 1;
        if (len > maxlen) {
          int leeway = (len - maxlen) / 2, q = len / 4;
          int d0 = dist(d, lo), d1 = dist(d, lo + q), d2 = dist(d, lo + 2 * q), d3 = dist(d, hi);
          int nl = lo;
          if (d0 > d3) nl += leeway;
          if (d1 > d2) nl += leeway;
          d.lo = imax(nl, lo);
          d.hi = imin(nl + maxlen - 1, hi);
        }
        hs.steps_wait = hp2;
        return false;
      }
      case WFA_HEURISTIC_XDROP: {
        if (hs.steps_wait > 0) return false;
        int cmax, ck, co;
        sw_max(d, score, cmax, ck, co);
        if (hs.max_sw_k != kDiagNull) {
          int mx = hs.max_sw_score, xd = hp0;
          auto keep = [&](int k) {
            bool ok;
            int sw = sw_score(d, k, score, ok);
            return ok && !(mx - sw >= xd);
          };
          int f = INT_MAX;
          for (int k = d.lo + lane; k <= d.hi; k += LW) if (keep(k)) { f = k; break; }
          int nlo = imin(G::min(f), d.hi + 1);
          int l = INT_MIN;
          for (int k = d.hi - lane; k >= nlo; k -= LW) if (keep(k)) { l = k; break; }
          int nhi = imax(G::max(l), nlo - 1);
          d.lo = nlo;
          d.hi = nhi;
          if (cmax > hs.max_sw_score) { hs.max_sw_score = cmax; hs.max_sw_k = ck; }
        } else {
          hs.max_sw_score = cmax;
          hs.max_sw_k = ck;
        }
        hs.steps_wait = hp1;
        return false;
      }
      case WFA_HEURISTIC_ZDROP: {
        if (hs.steps_wait > 0) return false;
        int cmax, ck, co;
        sw_max(d, score, cmax, ck, co);
        if (hs.max_sw_k == kDiagNull || cmax > hs.max_sw_score) {
          hs.max_sw_score = cmax; hs.max_wf_score = score; hs.max_sw_k = ck;
          hs.max_sw_off = co; hs.zdrop_last = score;
        } else if (hs.max_sw_score - cmax <= hp0) {
          hs.zdrop_last = score;
        } else if (score - hs.zdrop_last >= scope - 1) {
          return true;
        }
        hs.steps_wait = hp1;
        return false;
      }
      default:
        return false;
    }
  }

  // apply_heuristic_cutoff, src/aligner.rs:1644-1766.  True on a Z-drop.
  WFA_D bool apply_heuristic(int score) {
    WfD d = slot(CM, score);
    if (hk() == WFA_HEURISTIC_BANDED_STATIC && d.lo >= hp0 && d.hi <= hp1) return false;
    int lo_base = d.lo, hi_base = d.hi;
    const int32_t max_wf_base = hs.max_wf_score;
    bool z = heuristic_cutoff(d, score);
    // Corrected med/low keep the chain of a new Z-drop best cell (src/aligner.rs:1677-1688).
    if (PB && pgb && P.compat == WFA_COMPAT_CORRECTED && hs.max_wf_score == score && max_wf_base != score)
      m_bt(hs.max_sw_k, zd_pc, zd_pv);
    if (z) {
      end_score = hs.max_wf_score; end_k = hs.max_sw_k; end_off = hs.max_sw_off;
      return true;
    }
    if (lo_base > hi_base || (d.lo == lo_base && d.hi == hi_base)) return false;
    if (d.lo > d.hi) { d.flags |= kNullFlag; d.a = d.lo; d.b = d.hi; }
    WfD eq[NC];
    for (int c = 1; c < NC; ++c) eq[c] = slot(c, score);
    G::sync();
    put_ns(CM, score, d);
    if (AFF) {
      for (int c = 1; c < NC; ++c) {
        WfD w = eq[c];
        if (!wf_present(w)) continue;
        if (d.lo > w.lo) w.lo = d.lo;
        if (d.hi < w.hi) w.hi = d.hi;
        if (w.lo > w.hi) { w.flags |= kNullFlag; w.a = w.lo; w.b = w.hi; }
        put_ns(c, score, w);
      }
    }
    G::sync();
    return false;
  }

  // extend_end2end (src/aligner.rs:1004-1050) / extend_endsfree (:1053-1101).
  WFA_D bool extend_step(int score) {
    if (GEN && corr) return extend_step_corrected(score);
    WfD d = slot(CM, score);
    if (!wf_present(d)) {
      if (num_null_steps > scope) { status = WFA_STATUS_END_UNREACHABLE; return true; }
      return false;
    }
    int toff = 0;
    int tk = extend_wf(d, ef(), toff);
    if (ef()) {
      if (tk != INT_MAX) {
        end_score = score; end_k = tk; end_off = toff;
        status = WFA_STATUS_END_REACHED;
        return true;
      }
    } else {
      int ak = m - n;
      if (d.lo <= ak && ak <= d.hi && d.vals[ak - d.a] >= m) {
        end_score = score; end_k = ak; end_off = m;
        status = WFA_STATUS_END_REACHED;
        return true;
      }
    }
    if (hk() != WFA_HEURISTIC_NONE && apply_heuristic(score)) {
      status = WFA_STATUS_END_UNREACHABLE;
      return true;
    }
    return false;
  }

  // ---- BiWFA sub-aligner steps ---------------------------------------------------
  // init_alignment_component, src/aligner.rs:3205-3265: a single cell (k = 0,
  // offset 0) in component `comp` at score 0.
  WFA_D void init_alignment_component(int comp) {
    cscore = 0;
    cidx = 0;
    gstep = score_step_gcd();
    gphase = 0;
    gshift = 0;
    dscope = scope;
    for (int i = lane; i < scope * NC; i += LW) ws.ring[i] = wf_none();
    G::sync();
    hist_lo = -(n + scope + 2);
    hist_hi = m + scope + 2;
    num_null_steps = 0;
    status = WFA_STATUS_OK;
    end_score = 0; end_k = 0; end_off = 0;
    hs.steps_wait = (hk() == WFA_HEURISTIC_WFADAPTIVE || hk() == WFA_HEURISTIC_BANDED_ADAPTIVE) ? hp2
                    : (hk() == WFA_HEURISTIC_XDROP || hk() == WFA_HEURISTIC_ZDROP) ? hp1 : 0;
    hs.max_sw_score = 0; hs.max_wf_score = 0; hs.max_sw_k = kDiagNull;
    hs.max_sw_off = kOffsetNull; hs.zdrop_last = 0;
    hused = 0;
    int32_t* v = alloc(comp, 0, 0, 0);
    if (retry) return;
    if (lane == 0) v[0] = 0;
    WfD d;
    d.vals = v; d.lo = 0; d.hi = 0; d.a = 0; d.b = 0; d.flags = kPresent; d.adub = 0;
    put(comp, 0, d);
  }

  // One step of the score loop for a BiWFA sub-aligner: the compute step at
  // score s (s > 0), honouring the all-null scores, with null slots stored.
  WFA_D void bi_compute(int s) {
    advance();
    gphase = gphase + 1 == gstep ? 0 : gphase + 1;
    if (gphase != 0) {
      ++num_null_steps;
      for (int c = 0; c < NC; ++c) put_ns(c, s, wf_none());
      G::sync();
    } else {
      compute_step(s);
    }
  }

  // extend_biwfa_step, src/aligner.rs:3516-3554: extend M (with the maximum
  // antidiagonal when `max`), then the end test on `comp_end` and the
  // heuristic.  Returns true when done; max_ak as the reference reports it.
  WFA_D bool bi_extend(int score, bool max, int& max_ak) {
    max_ak = 0;
    WfD d = slot(CM, score);
    if (!wf_present(d)) {
      if (num_null_steps > scope) { status = WFA_STATUS_END_UNREACHABLE; return true; }
      return false;
    }
    int ak = 0;
    for (int k0 = d.lo + lane; k0 <= d.hi; k0 += LW * UNR) {
      // Offsets and first sequence words of UNR diagonals, then the rest.
      int32_t off[UNR], R[UNR];
      uint32_t x[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int k = k0 + u * LW;
        off[u] = k <= d.hi ? d.vals[k - d.a] : -1;
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int k = k0 + u * LW;
        R[u] = 0;
        x[u] = 0;
        if (off[u] >= 0) {
          R[u] = imin(n - (off[u] - k), m - off[u]);
          if (R[u] > 0) x[u] = pat.fetch(off[u] - k) ^ txt.fetch(off[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int k = k0 + u * LW;
        if (off[u] < 0) continue;
        if (R[u] > 0) {
          // lcp_fwd with its first compare done above
          int l;
          if (x[u]) {
            l = (int)((Warp::ffs(x[u]) - 1) / S::BITS);
          } else {
            l = S::UNITS;
            if (R[u] > S::UNITS)
              l += lcp_fwd(pat, off[u] - k + S::UNITS, txt, off[u] + S::UNITS, R[u] - S::UNITS);
          }
          off[u] += imin(l, R[u]);
          d.vals[k - d.a] = off[u];
        }
        ak = imax(ak, 2 * off[u] - k);
      }
    }
    ak = G::max(ak);
    if (lane == 0) slot(CM, score).adub = ak;
    G::sync();
    // check_component_termination, src/aligner.rs:3268-3302
    WfD e = slot(comp_end, score);
    int kend = m - n;
    if (wf_present(e) && kend >= e.lo && kend <= e.hi && rd(e, kend) >= m) {
      end_score = score; end_k = kend; end_off = m;
      status = WFA_STATUS_END_REACHED;
      return true;
    }
    if (hk() != WFA_HEURISTIC_NONE && apply_heuristic(score)) {
      status = WFA_STATUS_END_UNREACHABLE;
      return true;
    }
    max_ak = max ? ak : 0;
    return false;
  }

  // backtrace_affine_c, src/backtrace.rs:492-635: the classic backtrace over
  // every component's history (BiWFA base case), ending in `comp_end`.
  WFA_D void backtrace_affine_classic(int ascore, int k, int offset, int cend) {
    cg_end = cg_cap;
    cg_begin = cg_cap - 1;
    int matrix = cend;
    int score = ascore, v = offset - k, h = offset;
    if (cend == CM) {
      run('D', imax(n - v, 0));
      run('I', imax(m - h, 0));
    }
    constexpr int64_t I1O = 1, I1E = 2, I2O = 3, I2E = 4, D1O = 5, D1E = 6, D2O = 7, D2E = 8, MM = 9;
    while (v > 0 && h > 0 && score > 0 && status != WFA_STATUS_OOM) {
      int mis = score - P.mismatch;
      int go1 = score - P.o1 - P.e1, go2 = TWO ? score - P.o2 - P.e2 : -1;
      int ge1 = score - P.e1, ge2 = TWO ? score - P.e2 : -1;
      int64_t mx;
      if (matrix == CM) {
        int64_t misms = bt_pack(mis, k, 0, 1, MM, false, CM);
        int64_t mi1 = lmax(bt_pack(go1, k, -1, 1, I1O, true, CM), bt_pack(ge1, k, -1, 1, I1E, true, CI1));
        int64_t md1 = lmax(bt_pack(go1, k, 1, 0, D1O, false, CM), bt_pack(ge1, k, 1, 0, D1E, false, CD1));
        if (TWO) {
          int64_t mi2 = lmax(bt_pack(go2, k, -1, 1, I2O, true, CM), bt_pack(ge2, k, -1, 1, I2E, true, CI2));
          int64_t md2 = lmax(bt_pack(go2, k, 1, 0, D2O, false, CM), bt_pack(ge2, k, 1, 0, D2E, false, CD2));
          mx = lmax(misms, lmax(lmax(mi1, mi2), lmax(md1, md2)));
        } else {
          mx = lmax(misms, lmax(mi1, md1));
        }
      } else if (matrix == CI1) {
        mx = lmax(bt_pack(go1, k, -1, 1, I1O, true, CM), bt_pack(ge1, k, -1, 1, I1E, true, CI1));
      } else if (matrix == CD1) {
        mx = lmax(bt_pack(go1, k, 1, 0, D1O, false, CM), bt_pack(ge1, k, 1, 0, D1E, false, CD1));
      } else if (matrix == CI2) {
        mx = lmax(bt_pack(go2, k, -1, 1, I2O, true, CM), bt_pack(ge2, k, -1, 1, I2E, true, CI2));
      } else {
        mx = lmax(bt_pack(go2, k, 1, 0, D2O, false, CM), bt_pack(ge2, k, 1, 0, D2E, false, CD2));
      }
      if (mx < 0) break;
      if (matrix == CM) {
        int moff = (int)(mx >> 4);
        matches(offset - moff);
        offset = moff;
        v = offset - k; h = offset;
        if (v <= 0 || h <= 0) break;
      }
      int64_t t = mx & 0xF;
      if (t == MM) { score = mis; matrix = CM; }
      else if (t == I1O || t == D1O) { score = go1; matrix = CM; }
      else if (t == I2O || t == D2O) { score = go2; matrix = CM; }
      else if (t == I1E) { score = ge1; matrix = CI1; }
      else if (t == I2E) { score = ge2; matrix = CI2; }
      else if (t == D1E) { score = ge1; matrix = CD1; }
      else { score = ge2; matrix = CD2; }
      if (t == MM) { push('X'); offset -= 1; }
      else if (t == I1O || t == I1E || t == I2O || t == I2E) { push('I'); k -= 1; offset -= 1; }
      else { push('D'); k += 1; }
      v = offset - k; h = offset;
    }
    if (matrix == CM) {
      if (v > 0 && h > 0) {
        int nm = imin(v, h);
        matches(nm);
        v -= nm; h -= nm;
      }
      run('D', v);
      run('I', h);
    }
    cg_begin += 1;
    cg_score = ascore;
    G::sync();
  }

  // backtrace_components (src/aligner.rs:1489-1535): the BiWFA base case's.
  WFA_D void backtrace_components(int score, int k, int offset, int cend) {
    G::sync();
    if (AFF) {
      backtrace_affine_classic(score, k, offset, cend);
    } else {
      cg_end = cg_cap;
      cg_begin = cg_cap - 1;
      backtrace_linear(score, k, offset);
      cg_begin += 1;
      cg_score = score;
      G::sync();
    }
  }

  // ---- CIGAR output ------------------------------------------------------------
  WFA_D void run(uint8_t op, int cnt) {  // write_ops, src/backtrace.rs:689-698
    if (cnt <= 0) return;
    if (cg_begin - cnt + 1 < 0) { status = WFA_STATUS_OOM; cg_begin = -1; return; }
    for (int i = lane; i < cnt; i += LW) cg[cg_begin - i] = op;
    cg_begin -= cnt;
  }
  WFA_D void matches(int cnt) {  // write_matches, src/backtrace.rs:111-128
    if (cnt < 0) { cg_begin += -(int64_t)cnt; return; }
    run('M', cnt);
  }
  WFA_D void push(uint8_t op) { run(op, 1); }
  WFA_D uint8_t op_at(int64_t i) const { return cg[i]; }

  // M history lookup (st_m_offset, src/backtrace.rs:645-663; NULL cells ->
  // false, as outside the initialised range).
  WFA_D bool m_cell(int score, int k, int32_t& out) const {
    if (score < 0 || !has_slot(score)) return false;
    int4 r = ws.hist[(int64_t)score * hist_nc];
    if (!r.w || k < r.x || k > r.y) return false;
    out = ws.harena[r.z + (k - r.x)];
    return true;
  }
  WFA_D bool st_m_offset(int score, int k, int32_t& out) const {
    int32_t o;
    if (!m_cell(score, k, o) || o == kOffsetNull) return false;
    out = o;
    return true;
  }

  // backtrace_affine_singletrack, src/backtrace.rs:751-858
  WFA_D bool st_gap(int gscore, int l, int off_orig, int& k, int& offset) {
    int32_t mo;
    if (st_m_offset(gscore, k - l, mo) && mo + l >= off_orig && mo + l <= offset) {
      run('M', offset - (mo + l));
      run('I', l);
      k -= l;
      offset = mo;
      return true;
    }
    if (st_m_offset(gscore, k + l, mo) && mo >= off_orig && mo <= offset) {
      run('M', offset - mo);
      run('D', l);
      k += l;
      offset = mo;
      return true;
    }
    return false;
  }
  WFA_D void backtrace_singletrack(int ascore, int k, int offset) {
    int score = ascore, off_orig = offset;
    run('D', n - (offset - k));
    run('I', m - offset);
    bool in_m = true;
    int l = 0;
    while (score != 0 && status != WFA_STATUS_OOM) {
      if (in_m) {
        int v = offset - k, h = offset;
        int nm = lcp_bwd(pat, v, txt, h, imin(v, h));
        off_orig = offset - nm;
        int mis = score - P.mismatch;
        int32_t mo;
        if (st_m_offset(mis, k, mo) && mo == off_orig - 1) {
          run('M', nm);
          run('X', 1);
          offset = off_orig - 1;
          score = mis;
        } else {
          in_m = false;
          l = 0;
        }
      } else {
        ++l;
        int ind1 = score - P.o1 - l * P.e1;
        int ind2 = TWO ? score - P.o2 - l * P.e2 : -1;
        if (st_gap(ind1, l, off_orig, k, offset)) { score = ind1; in_m = true; }
        else if (st_gap(ind2, l, off_orig, k, offset)) { score = ind2; in_m = true; }
        else if (ind1 < 0 && ind2 < 0) break;
      }
    }
    int v = offset - k, h = offset;
    int nm = imin(v, h);
    v -= nm;
    h -= nm;
    run('M', nm);
    run('D', v);
    run('I', h);
  }

  // backtrace_linear, src/backtrace.rs:132-258
  // Backtrace lookups of src/backtrace.rs:44-330 (bt_misms: dk 0; bt_ins*: dk
  // -1, cell k-1; bt_del*: dk +1, cell k+1) on component c of the history:
  // the packed (offset << 4 | type), or OFFSET_NULL outside the initialised
  // range / for a missing wavefront.
  WFA_D int64_t bt_pack(int score, int k, int dk, int add, int64_t type, bool ins, int c = CM) const {
    if (score < 0) return kOffsetNull;
    int4 r = ws.hist[(int64_t)score * hist_nc + c];
    if (!r.w) return kOffsetNull;
    bool inside;
    if (dk == 0) inside = r.x <= k && k <= r.y;
    else if (ins) inside = r.x < k && k - 1 <= r.y;
    else inside = r.x <= k + 1 && k < r.y;
    if (!inside) return kOffsetNull;
    int32_t o = ws.harena[r.z + (k + dk - r.x)];
    return ((int64_t)(o + add) << 4) | type;
  }
  WFA_D void backtrace_linear(int ascore, int k, int offset) {
    int score = ascore, v = offset - k, h = offset;
    if (v < n) run('D', n - v);
    if (h < m) run('I', m - h);
    const bool indel = P.metric == WFA_METRIC_INDEL;
    while (v > 0 && h > 0 && score > 0 && status != WFA_STATUS_OOM) {
      int ms = score - P.mismatch, gs = score - P.o1;
      int64_t misms = indel ? (int64_t)kOffsetNull : bt_pack(ms, k, 0, 1, 9, false);
      int64_t ins = bt_pack(gs, k, -1, 1, 1, true);
      int64_t del = bt_pack(gs, k, 1, 0, 5, false);
      int64_t mx = lmax(misms, lmax(ins, del));
      if (mx < 0) break;
      int moff = (int)(mx >> 4);
      matches(offset - moff);
      offset = moff;
      v = offset - k; h = offset;
      if (v <= 0 || h <= 0) break;
      int t = (int)(mx & 0xF);
      if (t == 9) { score = ms; push('X'); offset -= 1; }
      else if (t == 1) { score = gs; push('I'); k -= 1; offset -= 1; }
      else { score = gs; push('D'); k += 1; }
      v = offset - k; h = offset;
    }
    if (v > 0 && h > 0) {
      int nm = imin(v, h);
      matches(nm);
      v -= nm; h -= nm;
    }
    run('D', v);
    run('I', h);
  }

  // Forward CIGAR writes of the unpack: at most `limit` (exclusive) -- the
  // chain operations not yet read sit above it in the same slot.
  WFA_D bool fwd(int64_t& p, int64_t limit, uint8_t op, int cnt) {
    if (cnt <= 0) return true;
    if (p + cnt > limit) { status = WFA_STATUS_OOM; return false; }
    for (int i = lane; i < cnt; i += LW) cg[p + i] = op;
    p += cnt;
    return true;
  }
  // ---- med/low: the chain of packed CIGARs -------------------------------------
  // backtrace_piggyback_bt (src/aligner.rs:1463-1486): traceback_from
  // (src/bt_buffer.rs:196-212) collects the chain's packed CIGARs back to
  // its initial block; unpack_piggyback (src/aligner.rs:232-311) then spells
  // them from the first.  The end cell's own packed CIGAR stays in a
  // register; the offloaded blocks (each of at least 9 operations: only
  // packed CIGARs at least half full are offloaded) are stored 4 bytes each
  // backwards from the end of the pair's CIGAR slot and read from the first
  // while the CIGAR is written forwards from the slot's start: at most
  // 2 (n + m) / 9 blocks take less than the (n + m + 1) bytes the CIGAR
  // leaves free, so the unread blocks always lie above the write point.
  WFA_D uint32_t cg_word(int64_t i) const {
    return (uint32_t)cg[i] | ((uint32_t)cg[i + 1] << 8) | ((uint32_t)cg[i + 2] << 16) | ((uint32_t)cg[i + 3] << 24);
  }
  // The operations of one packed CIGAR, matches re-extended before each
  // (only in M when affine, where an X after I/D is the gap close and is
  // dropped); writes below `limit`.
  WFA_D bool unpack_block(uint32_t pcig, int64_t& p, int64_t limit, int& v, int& h, bool& in_m) {
    const bool affine = AFF;
    int length = kPcMaxLength;
    if (pcig < kPcFullMask) {
      const int fr = pcig ? (int)Warp::clz(pcig) / 2 : kPcMaxLength;
      length -= fr;
      pcig = fr >= kPcMaxLength ? 0u : pcig << (2 * fr);
    }
    for (int j = 0; j < length; ++j) {
      if (in_m || !affine) {
        const int nm = lcp_fwd(pat, v, txt, h, imax(0, imin(n - v, m - h)));
        if (!fwd(p, limit, 'M', nm)) return false;
        v += nm;
        h += nm;
      }
      const uint32_t op = pcig >> 30;
      pcig <<= 2;
      const uint8_t ch = op == kPcDel ? 'D' : op == kPcMisms ? 'X' : op == kPcIns ? 'I' : '?';
      if (affine && !in_m && ch == 'X') { in_m = true; continue; }
      if (!fwd(p, limit, ch, 1)) return false;
      v += (op == kPcDel || op == kPcMisms) ? 1 : 0;
      h += (op == kPcIns || op == kPcMisms) ? 1 : 0;
      in_m = op == kPcMisms || op == 0;
    }
    return true;
  }
  WFA_D void backtrace_pb(uint32_t pc, uint32_t pv, int score, int k, int offset) {
    cg_begin = 0;
    cg_end = 0;
    cg_score = score;
    const uint32_t end_pc = pc;
    int64_t rdp = cg_cap;
    int32_t guard = 0;
    uint32_t init = 0;
    for (;;) {
      if (pv == kBtNull || ++guard > bt_used + 1) { status = WFA_STATUS_OOM; return; }
      const uint2 blk = ws.bt[pv];
      if (blk.y == kBtNull) { init = blk.x; break; }  // the initial block: its position's index
      if (rdp < 4) { status = WFA_STATUS_OOM; return; }
      rdp -= 4;
      if (lane == 0)
        for (int b = 0; b < 4; ++b) cg[rdp + b] = (uint8_t)(blk.x >> (8 * b));
      pv = blk.y;
    }
    G::sync();
    const int2 ip = ws.btinit[init];
    int64_t p = 0;
    int v = ip.x, h = ip.y;
    if (!fwd(p, rdp, 'I', h) || !fwd(p, rdp, 'D', v)) return;
    bool in_m = true;
    for (int64_t b = rdp; b < cg_cap; b += 4) {
      const uint32_t pcig = cg_word(b);
      G::sync();  // every lane has read the block before it may be overwritten
      if (!unpack_block(pcig, p, b + 4, v, h, in_m)) return;
    }
    if (!unpack_block(end_pc, p, cg_cap, v, h, in_m)) return;
    // As the reference, a negative count (end behind the unpacked position) moves back.
    const int nm = imin(offset - k - v, offset - h);
    if (!fwd(p, cg_cap, 'M', nm)) return;
    v += nm;
    h += nm;
    if (!fwd(p, cg_cap, 'I', m - h) || !fwd(p, cg_cap, 'D', n - v)) return;
    cg_end = p;
  }
  // The end cell of the current score's M (backtrace_piggyback,
  // src/aligner.rs:1443-1459): no CIGAR without an M at that score.
  WFA_D void backtrace_pb_current(int score, int k, int offset) {
    if (!mbase) { cg_begin = 0; cg_end = 0; cg_score = score; return; }
    uint32_t c, v;
    m_bt(k, c, v);
    backtrace_pb(c, v, score, k, offset);
  }
  // The Z-drop end (backtrace_zdrop_end, :1393-1411).
  WFA_D void backtrace_zdrop(int score) {
    if (PB && pgb && P.compat == WFA_COMPAT_CORRECTED) {
      G::sync();
      backtrace_pb(zd_pc, zd_pv, end_score, end_k, end_off);
      G::sync();
      return;
    }
    backtrace_from(zdrop_from(score), end_k, end_off);
  }

  WFA_D void backtrace_from(int score, int k, int offset) {  // src/aligner.rs:1414-1436
    G::sync();
    if (PB && pgb) {
      backtrace_pb_current(score, k, offset);
      G::sync();
      return;
    }
    cg_end = cg_cap;
    cg_begin = cg_cap - 1;
    if (AFF) backtrace_singletrack(score, k, offset);
    else backtrace_linear(score, k, offset);
    cg_begin += 1;
    cg_score = score;
    G::sync();
  }

  // ---- CIGAR post-processing: src/cigar.rs, src/aligner.rs:1545-1640 ----------
  WFA_D int32_t score_classic(int64_t b, int64_t e) const {  // score_gap_* with user penalties
    const int32_t* p = P.orig;
    int32_t s = 0;
    if (CLS == kEditClass) {
      for (int64_t i = b; i < e; ++i) s += op_at(i) != 'M';
      return s;
    }
    if (CLS == kLinearClass) {
      for (int64_t i = b; i < e; ++i) {
        uint8_t op = op_at(i);
        s -= op == 'M' ? p[0] : op == 'X' ? p[1] : p[2];
      }
      return s;
    }
    if (CLS == kAffineClass) {
      uint8_t last = 0;
      for (int64_t i = b; i < e; ++i) {
        uint8_t op = op_at(i);
        if (op == 'M') s -= p[0];
        else if (op == 'X') s -= p[1];
        else s -= p[3] + (last == op ? 0 : p[2]);
        last = op;
      }
      return s;
    }
    int64_t i = b;
    while (i < e) {
      uint8_t op = op_at(i);
      int64_t j = i;
      while (j < e && op_at(j) == op) ++j;
      int32_t len = (int32_t)(j - i);
      if (op == 'M') s -= p[0] * len;
      else if (op == 'X') s -= p[1] * len;
      else s -= imin(p[2] + p[3] * len, p[4] + p[5] * len);
      i = j;
    }
    return s;
  }
  WFA_D int32_t cigar_wfa_score(int64_t b, int64_t e, int v, int h) const {  // :2700-2719
    int32_t c = score_classic(b, e);
    if (CLS == kEditClass) return c;
    if (P.match < 0) return -P.match * (v + h) - 2 * c;
    return -c;
  }
  WFA_D int cigar_skip_gap(uint8_t op, int maxlen) {  // :1580-1592
    int len = 0;
    while (len < maxlen && cg_begin < cg_end && op_at(cg_begin) == op) { ++cg_begin; ++len; }
    return len;
  }
  // maxtrim_gap_linear / _affine / _affine2p (src/cigar.rs:207-444); returns trimmed.
  WFA_D bool maxtrim_ops() {
    int64_t b = cg_begin, e = cg_end;
    if (b >= e) return false;
    const int32_t* p = P.orig;
    int32_t max_score = 0, mv = 0, mh = 0, s = 0, v = 0, h = 0;
    int64_t max_off = b;
    if (CLS != kAffine2pClass) {
      int32_t match_score = p[0] != 0 ? p[0] : -1;
      uint8_t last = 0;
      for (int64_t i = b; i < e; ++i) {
        uint8_t op = op_at(i);
        if (op == 'M') { s -= match_score; ++v; ++h; }
        else if (op == 'X') { s -= p[1]; ++v; ++h; }
        else if (op == 'I') { s -= CLS == kLinearClass ? p[2] : p[3] + (last == 'I' ? 0 : p[2]); ++h; }
        else if (op == 'D') { s -= CLS == kLinearClass ? p[2] : p[3] + (last == 'D' ? 0 : p[2]); ++v; }
        last = op;
        if (max_score < s) { max_score = s; max_off = i; mv = v; mh = h; }
      }
    } else {
      uint8_t last = 0;
      int32_t len = 0;
      auto opsc = [&](uint8_t op, int32_t L) -> int32_t {
        if (op == 'M') { v += L; h += L; return (p[0] != 0 ? p[0] : -1) * L; }
        if (op == 'X') { v += L; h += L; return p[1] * L; }
        if (op == 'D') { v += L; return imin(p[2] + p[3] * L, p[4] + p[5] * L); }
        if (op == 'I') { h += L; return imin(p[2] + p[3] * L, p[4] + p[5] * L); }
        return 0;
      };
      for (int64_t i = b; i < e; ++i) {
        uint8_t op = op_at(i);
        if (op != last && last != 0) {
          s -= opsc(last, len);
          len = 0;
          if (max_score < s) { max_score = s; max_off = i - 1; mv = v; mh = h; }
        }
        last = op;
        ++len;
      }
      s -= opsc(last, len);
      if (max_score < s) { max_score = s; max_off = e - 1; mv = v; mh = h; }
    }
    bool trimmed = max_off != e - 1;
    if (max_score == 0) {
      cg_begin = 0; cg_end = 0; cg_score = INT_MIN; cg_ev = -1; cg_eh = -1;
    } else {
      cg_end = max_off + 1; cg_score = max_score; cg_ev = mv; cg_eh = mh;
    }
    return trimmed;
  }
  WFA_D bool maxtrim_cigar() {  // src/aligner.rs:1545-1577
    if (CLS == kEditClass) return false;
    int bv = 0, bh = 0;
    if (ef()) {
      bh = cigar_skip_gap('I', t0);
      if (bh == 0) bv = cigar_skip_gap('D', p0);
    }
    if (cg_begin >= cg_end) {
      cg_begin = 0; cg_end = 0; cg_score = INT_MIN; cg_ev = -1; cg_eh = -1;
      return true;
    }
    bool trimmed = maxtrim_ops();
    if (cg_score != INT_MIN) {
      cg_score = cigar_wfa_score(cg_begin, cg_end, cg_ev, cg_eh);
      cg_begin -= bv + bh;
      cg_ev += bv;
      cg_eh += bh;
    }
    return trimmed;
  }
  WFA_D int32_t rescore_heuristic(int score) {  // src/aligner.rs:1605-1640
    if (hk() == WFA_HEURISTIC_NONE || !AFF) return score;
    int64_t b = cg_begin, e = cg_end;
    if (ef()) {
      int trailing = (n - cg_ev) + (m - cg_eh);
      // end.saturating_sub(trailing as usize): negative wraps, view empty.
      cg_end = (trailing < 0 || e - trailing < 0) ? 0 : e - trailing;
      uint8_t op = b < cg_cap ? op_at(b) : 0;
      int fr = op == 'I' ? t0 : op == 'D' ? p0 : 0;
      cigar_skip_gap(op, fr);
    }
    int64_t vb = cg_begin, ve = cg_end > vb ? cg_end : vb;
    int32_t r = 0;
    if (ve > vb) {
      int v = 0, h = 0;
      for (int64_t i = vb; i < ve; ++i) { v += op_at(i) != 'I'; h += op_at(i) != 'D'; }
      r = cigar_wfa_score(vb, ve, v, h);
    }
    cg_begin = b;
    cg_end = e;
    cg_score = r;
    return r;
  }

  // The score a Z-drop end is backtraced from (backtrace_zdrop_end,
  // src/aligner.rs:1393-1411): C reads med/low at the current score (where
  // the cell may be dead), high memory at the best cell's score; Corrected
  // reads every mode at the best cell's score.
  WFA_D int zdrop_from(int score) const {
    if (GEN && P.compat == WFA_COMPAT_CORRECTED) return end_score;
    return end_score >= 0 && !(PB && pgb) ? end_score : score;
  }

  // ---- one pair: align_end2end_span (src/aligner.rs:638-698) and
  // align_endsfree (:707-831), C compatibility ----------------------------------
  // The score loop as begin() / step() / finish(): step() runs the loop from
  // the extend of one score that can hold a wavefront (a multiple of gstep)
  // through the next such score's compute, with the all-null scores between.
  // align() is begin(), steps until one returns true, finish().
  int32_t cur;  // the score loop's current score
  WFA_D void begin() {
    retry = false;
    hused = 0;
    cg_begin = 0; cg_end = 0; cg_score = INT_MIN; cg_ev = -1; cg_eh = -1;
    init_alignment();
    cur = 0;
  }
  // One step of the score loop; true when the loop is over (status set, or
  // retry).
  WFA_D bool step() {
    const int hard_limit = 1 << 26;  // no reference alignment runs this long
    int score = cur;
    for (;;) {
      bool done;
      if (gphase != 0) {  // all-null score: no M to extend (extend_end2end, null branch)
        if (GEN && corr && c_has && c_total <= score) {
          // Corrected: the candidate is final once the score reaches its
          // total; null steps do not end the search while one is pending.
          done = true;
          end_score = c_score; end_k = c_k; end_off = c_off;
          status = WFA_STATUS_END_REACHED;
        } else {
          done = !(GEN && corr && c_has) && num_null_steps > scope;
          if (done) status = WFA_STATUS_END_UNREACHABLE;
        }
        if (!modular && !(PB && pgb)) {
          if ((int64_t)(score + 1) * hist_nc > P.hist_scores) { retry = true; break; }
          if (lane == 0)
            for (int c = 0; c < hist_nc; ++c) ws.hist[(int64_t)score * hist_nc + c] = int4{1, 0, 0, 0};
        }
      } else {
        done = extend_step(score);
        hist_commit(score);
      }
      if (done || retry) break;
      ++score;
      advance();
      gphase = gphase + 1 == gstep ? 0 : gphase + 1;
      if (!has_slot(score)) { status = WFA_STATUS_MAX_STEPS_REACHED; break; }
      const bool computed = gphase == 0;
      if (computed) {
        compute_step(score);
      } else {
        ++num_null_steps;
        if (PB && pgb) mbase = nullptr;
      }
      if (retry) break;
      if (score >= P.max_steps || score >= hard_limit) { status = WFA_STATUS_MAX_STEPS_REACHED; break; }
      // probe_bt_buffer (src/aligner.rs:479-513): compact the backtrace
      // buffer every PROBE_INTERVAL_COMPACT scores while it holds more than
      // max_memory_compact bytes (8 per block).
      if (PB && pgb && score % P.bt_probe == 0 && (int64_t)bt_used * 8 > P.bt_limit) {
        compact_bt();
        if (retry) break;
      }
      if (computed) { cur = score; return false; }
    }
    cur = score;
    return true;
  }
  WFA_D int32_t align() {
    begin();
    if (!retry)
      while (!step()) {
      }
    return finish();
  }
  // After the score loop: backtrace, CIGAR post-processing and the status.
  WFA_D int32_t finish() {
    const int32_t score = cur;
    if (retry) { status = kStatusRetry; return 0; }
    int32_t result = score;
    const bool cigar = P.compute_alignment != 0;
    if (!ef()) {
      if (status == WFA_STATUS_END_REACHED) {
        if (cigar) {
          backtrace_from(score, end_k, end_off);
          cg_ev = end_off - end_k;
          cg_eh = end_off;
          result = rescore_heuristic(score);
        }
        if (status != WFA_STATUS_OOM) status = WFA_STATUS_COMPLETED;
      } else if (status == WFA_STATUS_END_UNREACHABLE && end_off != kOffsetNull) {
        if (cigar) {
          backtrace_zdrop(score);
          maxtrim_cigar();
        }
        if (status != WFA_STATUS_OOM) status = WFA_STATUS_PARTIAL;
      }
    } else if (status == WFA_STATUS_END_REACHED || status == WFA_STATUS_END_UNREACHABLE) {
      bool unreachable = status == WFA_STATUS_END_UNREACHABLE;
      // Corrected mode: the candidate's cell can be from an earlier score,
      // and its total is the alignment's score (src/aligner.rs:772-777).
      const bool cand = GEN && corr && c_has && !unreachable;
      if (cand) result = c_total;
      if (cigar && (status == WFA_STATUS_END_REACHED || end_off != kOffsetNull)) {
        if (cand && PB && pgb) {
          G::sync();
          backtrace_pb(cand_pc, cand_pv, c_score, c_k, c_off);
          G::sync();
        } else if (cand) {
          backtrace_from(c_score, c_k, c_off);
        } else if (unreachable) {
          backtrace_zdrop(score);
        } else {
          backtrace_from(score, end_k, end_off);
        }
        if (cand) cg_score = c_total;
        if (status == WFA_STATUS_OOM) return result;
        if (P.extension || unreachable) {
          bool trimmed = maxtrim_cigar();
          status = (trimmed || unreachable) ? WFA_STATUS_PARTIAL : WFA_STATUS_COMPLETED;
        } else {
          cg_ev = end_off - end_k;
          cg_eh = end_off;
          if (!cand) result = rescore_heuristic(score);
          status = WFA_STATUS_COMPLETED;
        }
      } else {
        status = unreachable ? WFA_STATUS_PARTIAL : WFA_STATUS_COMPLETED;
      }
    }
    return result;
  }
};

// Per-pair set-up of an aligner A (its workspace and lane already set) for
// pair `pair` of the launch.
template <int CLS, class S, bool GEN, int LW, bool PB>
WFA_D void setup_pair(PairAligner<CLS, S, GEN, 1, LW, PB>& A, const AlignParams& P, int64_t pair, S pat,
                      S txt) {
  A.pat = pat;
  A.txt = txt;
  A.n = P.p_len[pair];
  A.m = P.t_len[pair];
  A.scope = P.scope;
  A.wmax = P.wmax;
  A.compact = P.ring_slots > 0;
  A.modular = P.compute_alignment == 0;
  A.pgb = PB && !A.modular && P.piggyback != 0;
  // Med/low components are modular: no score cap.
  A.cap = A.modular || A.pgb ? INT_MAX : imax(A.dims_num(1000, 1000), A.dims_num(A.n, A.m));
  A.endsfree = P.span == WFA_SPAN_ENDSFREE;
  A.hkind = P.hkind; A.hp0 = P.hp0; A.hp1 = P.hp1; A.hp2 = P.hp2;
  A.hist_nc = 1;
  // Med/low: each cell's pcigar and block index sit ring_slots x wmax and
  // twice that many words after its offset (the ring lies in the scratch
  // slice, three arrays of the same shape).
  A.pcoff = (int64_t)P.ring_slots * P.wmax;
  A.mbase = nullptr;
  A.keep_null_slots = false;
  A.comp_end = CM;
  if (P.extension) { A.p0 = 0; A.pf = A.n; A.t0 = 0; A.tf = A.m; }
  else if (A.endsfree) { A.p0 = P.p0; A.pf = P.pf; A.t0 = P.t0; A.tf = P.tf; }
  else { A.p0 = A.pf = A.t0 = A.tf = 0; }
  A.cg = nullptr;
  A.cg_cap = 0;
  if (!A.modular && P.cigars) {
    A.cg = P.cigars + P.cigar_off[pair];
    A.cg_cap = 2 * ((int64_t)A.n + A.m) + 1;
  }
}

// The result record of an aligned pair (lane 0 of the group writes it).
template <int CLS, class S, bool GEN, int LW, bool PB>
WFA_D void write_result(const PairAligner<CLS, S, GEN, 1, LW, PB>& A, const AlignParams& P, int64_t pair,
                        int32_t score) {
  if (A.lane == 0) {
    wfa_result_t r;
    r.score = score;
    r.status = A.status;
    bool has = A.cg_end > A.cg_begin && !A.modular;
    r.cigar_begin = has ? (int32_t)A.cg_begin : 0;
    r.cigar_length = has ? (int32_t)(A.cg_end - A.cg_begin) : 0;
    r.cigar_score = A.cg_score;
    r.end_v = A.cg_ev;
    r.end_h = A.cg_eh;
    r.end_score = A.end_score;
    r.end_k = A.end_k;
    r.end_offset = A.end_off;
    P.results[pair] = r;
  }
}

// Set up and align pair `pair` of the launch with workspace `ws`, writing
// its result.  Returns true if the pair must be retried with more scratch.
template <int CLS, class S, bool GEN = true, int LW = WFA_WARP, bool PB = false>
WFA_D bool align_one(const AlignParams& P, const Workspace& ws, int64_t pair, S pat, S txt) {
  PairAligner<CLS, S, GEN, 1, LW, PB> A(P);
  A.ws = ws;
  A.lane = Lanes<LW>::lane();
  setup_pair(A, P, pair, pat, txt);
  int32_t score = A.align();
  if (A.status == kStatusRetry) return true;
  write_result(A, P, pair, score);
  return false;
}

}  // namespace wfab
