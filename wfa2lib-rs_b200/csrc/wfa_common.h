// wfa_common.h -- types shared by the host side and the kernels.
#pragma once
#include <stdint.h>

#include "../../include/wfa_b200.h"

namespace wfab {

// PROBE_INTERVAL_COMPACT (src/aligner.rs:360): scores between the med/low
// backtrace buffer's compaction probes.
constexpr int32_t kProbeIntervalCompact = 6000;

// OFFSET_NULL (src/offset.rs:15) and DPMATRIX_DIAGONAL_NULL (:46).
constexpr int32_t kOffsetNull = INT32_MIN / 2;
constexpr int32_t kDiagNull = INT32_MAX;

// Internal pair status: the pair needs more scratch than this launch gave it
// and is re-run by the host with a larger configuration.
constexpr int32_t kStatusRetry = 100;

// Metric classes compiled as separate kernel instantiations.
enum MetricClass { kEditClass = 0, kLinearClass = 1, kAffineClass = 2, kAffine2pClass = 3 };

// Everything a launch needs; passed by value (kernel parameter space).
struct AlignParams {
  // Metric and internal penalties (after the Eizenga transform,
  // src/penalties.rs:157-296); orig = user penalties for CIGAR scoring.
  int32_t metric;
  int32_t match, mismatch, o1, e1, o2, e2;
  int32_t orig[6];
  int32_t scope;  // max_score_scope (src/components.rs:435-505)
  // Span: 0 end-to-end, 1 ends-free.  extension: free ends = whole lengths.
  int32_t span, extension;
  int32_t p0, pf, t0, tf;
  // Heuristic (wfa_heuristic_kind_t and its three parameters).
  int32_t hkind, hp0, hp1, hp2;
  int32_t compute_alignment;
  // Med/low memory with an alignment -- the piggyback backtrace: 1 med,
  // 2 low (0: neither).  Its backtrace buffer per lane group: bt_cap blocks,
  // bt_init_cap initial positions, compacted above bt_limit bytes
  // (max_memory_compact).
  int32_t piggyback;
  int32_t bt_cap, bt_init_cap;
  int64_t bt_limit;
  int32_t bt_probe;  // scores between compaction probes (PROBE_INTERVAL_COMPACT, 6000)
  // Compat: 0 C (reproduce C's known bugs), 1 Corrected (src/aligner.rs:53-94).
  int32_t compat;
  int32_t max_steps;
  // BiWFA growth-phase I/D rings (BiDriver::find_breakpoint): 0 as chosen
  // by the search's length; 1 (tests) kept until the overlap scans, so that
  // every search restarts; 2 off.
  int32_t bi_idc;
  // Input.
  int32_t format;  // wfa_seq_format_t
  const uint8_t* seq;
  int64_t seq_bytes;
  const int64_t* p_off;
  const int32_t* p_len;
  const int64_t* t_off;
  const int32_t* t_len;
  const int64_t* cigar_off;
  uint8_t* cigars;
  wfa_result_t* results;
  const int64_t* pair_list;  // NULL: pairs 0..num_pairs-1
  int64_t num_pairs;
  // Scratch (one slice per resident warp).
  int32_t* scratch;
  int64_t warp_words;  // ints per warp slice
  int32_t wmax;        // ring slot width (cells)
  // Compact ring of the unidirectional aligner: slots per lane group (0: the
  // full [scope][components] ring) and the width of the device-memory ring
  // that takes rows wider than wmax (0: none).
  int32_t ring_slots;
  int32_t wspill;
  // Depth (scores) of the descriptor ring of the unidirectional aligner: the
  // scope, or with the compact layout and a power-of-two score step the
  // scores of the scope that can hold a wavefront (0: the scope).
  int32_t desc_depth;
  int32_t wmax_base;   // BiWFA base-case ring slot width (cells)
  int32_t ring_smem;   // 1: ring cells in shared memory (else in the scratch slice)
  int32_t seq_smem_words;  // per sequence staged in shared memory (0: none)
  int32_t max_len_sum;     // longest n + m of the launch
  int32_t hist_scores; // M history capacity (scores)
  int64_t hist_words;  // M history arena capacity (cells)
  int64_t dom_words;   // Corrected-mode dominance array per warp (cells; 0: none)
  unsigned long long* work_counter;
  int32_t* retry_count;
  // Device-checks build (WFA_DEVICE_CHECKS): failed index checks counted here.
  int32_t* check_count;
};

// Score step of the unidirectional aligner: scores that are not multiples
// of it hold no wavefront (the gcd of the recurrences' score offsets and, with
// begin-free seeds of a match reward, of the seed scores).  The same rule as
// PairAligner::score_step_gcd, for sizing the compact ring on the host.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int score_gcd(int a, int b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) { int t = a % b; a = b; b = t; }
  return a;
}
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int score_step(const AlignParams& P, int cls) {
  int g;
  if (cls == kEditClass) g = 1;
  else if (cls == kLinearClass) g = score_gcd(P.mismatch, P.o1);
  else g = score_gcd(score_gcd(P.mismatch, P.o1 + P.e1), P.e1);
  if (cls == kAffine2pClass) g = score_gcd(score_gcd(g, P.o2 + P.e2), P.e2);
  const bool ef = P.span == WFA_SPAN_ENDSFREE;
  const int p0 = P.extension ? 0 : P.p0, t0 = P.extension ? 0 : P.t0;
  if (ef && P.match != 0 && (p0 > 0 || t0 > 0)) g = score_gcd(g, -P.match);
  return g < 1 ? 1 : g;
}
// log2 of a power-of-two score step, else 0 (the descriptor ring then keeps
// one slot per score).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int score_shift(int g) {
  int k = 0;
  while ((1 << k) < g) ++k;
  return (1 << k) == g ? k : 0;
}
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int compact_desc_depth(const AlignParams& P, int cls) {
  return ((P.scope - 1) >> score_shift(score_step(P, cls))) + 1;
}
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int bi_idc_rows(int nc, int e1, int e2) {
  // BiWFA's growth phase keeps its I/D rows in a ring of their own after the
  // scope x NC rows: e + 1 rows for each of I and D of a piece.
  return nc >= 3 ? 2 * (e1 + 1) + (nc == 5 ? 2 * (e2 + 1) : 0) : 0;
}
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int compact_ring_slots(const AlignParams& P, int cls) {
  const int g = score_step(P, cls);
  int slots = (P.scope - 1) / g + 1;
  if (cls >= kAffineClass) slots += 2 * (P.e1 / g + 1);
  if (cls == kAffine2pClass) slots += 2 * (P.e2 / g + 1);
  return slots;
}

}  // namespace wfab
