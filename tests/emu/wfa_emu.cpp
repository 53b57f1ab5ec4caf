// wfa_emu.cpp -- TEST-ONLY host builds of the device aligner (wfa_align.cuh).
// Default build: a one-lane warp.  With -DWFA_EMU_THREADS: 32 host threads
// per warp (WFA_EMU_LANES=8: an 8-lane group), __syncwarp and the reductions
// as barriers.  The CPU tests compare
// them with the oracle so the kernel's logic is checked before it runs on a
// GPU.  Not part of the product.
#define WFA_EMU 1
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../wfa2lib-rs_b200/csrc/wfa_align.cuh"
#include "../../wfa2lib-rs_b200/csrc/wfa_biwfa.cuh"
#include "../../wfa2lib-rs_b200/csrc/wfa_params.h"

using namespace wfab;

#ifdef WFA_EMU_THREADS
namespace wfab {
thread_local int g_emu_lane = 0;
EmuWarp* g_emu_warp = nullptr;
}  // namespace wfab
#endif

template <int CLS, bool GEN, bool PB>
static bool run_lane_g(const AlignParams& P, const Workspace& ws, int64_t i) {
  if (P.format == WFA_SEQ_PACKED2) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(P.seq);
    SeqPacked sp{w + P.p_off[i], P.p_len[i], (P.p_len[i] + 15) >> 4};
    SeqPacked st{w + P.t_off[i], P.t_len[i], (P.t_len[i] + 15) >> 4};
    return align_one<CLS, SeqPacked, GEN, WFA_WARP, PB>(P, ws, i, sp, st);
  }
  SeqAscii sp{P.seq + P.p_off[i], P.p_len[i]};
  SeqAscii st{P.seq + P.t_off[i], P.t_len[i]};
  return align_one<CLS, SeqAscii, GEN, WFA_WARP, PB>(P, ws, i, sp, st);
}

// Same dispatch as the kernel launcher: the lean instantiation for
// end-to-end alignments without a heuristic, the med/low one for med/low
// with an alignment, the general one otherwise.
template <int CLS>
static bool run_lane(const AlignParams& P, const Workspace& ws, int64_t i) {
  if (P.piggyback && P.compute_alignment) return run_lane_g<CLS, true, true>(P, ws, i);
  if (P.span == WFA_SPAN_END2END && P.hkind == WFA_HEURISTIC_NONE)
    return run_lane_g<CLS, false, false>(P, ws, i);
  return run_lane_g<CLS, true, false>(P, ws, i);
}

// The kernel's compact ring: P.ring_slots slots of P.wmax cells (narrow, as
// the shared-memory slots are), rows wider than that in the spill ring of
// P.wspill cells per slot -- both paths run in every emulated alignment.
// Med/low: the ring as wide as any wavefront, with the pcigar and block
// arrays after the offsets, and the backtrace buffer.
template <int CLS>
static bool run_pair(const AlignParams& P, int64_t i) {
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const size_t arrays = P.piggyback ? 3 : 1;
  std::vector<WfD> ring((size_t)P.desc_depth * NC);
  std::vector<int32_t> ringv(arrays * P.ring_slots * P.wmax, 0x5A5A5A5A);
  std::vector<int32_t> ringg((size_t)P.ring_slots * P.wspill, 0x5A5A5A5A);
  std::vector<int4> hist((size_t)P.hist_scores, int4{0, -1, 0, 0});
  std::vector<int32_t> harena((size_t)P.hist_words, 0x5A5A5A5A);
  std::vector<int32_t> dom((size_t)P.dom_words, 0x5A5A5A5A);
  std::vector<uint2> bt((size_t)P.bt_cap, uint2{0x5A5A5A5A, 0x5A5A5A5A});
  std::vector<int2> btinit((size_t)P.bt_init_cap, int2{0x5A5A5A5A, 0x5A5A5A5A});
  std::vector<uint32_t> btmark(2 * (((size_t)P.bt_cap + 31) / 32) + 1, 0x5A5A5A5A);
  Workspace ws{ring.data(), ringv.data(), hist.data(), harena.data(),
               P.dom_words ? dom.data() : nullptr, ringg.data(), bt.data(), btinit.data(), btmark.data()};
#ifdef WFA_EMU_THREADS
  EmuWarp warp;
  g_emu_warp = &warp;
  bool retry[WFA_WARP];
  std::vector<std::thread> lanes;
  for (int l = 0; l < WFA_WARP; ++l)
    lanes.emplace_back([&, l]() {
      g_emu_lane = l;
      retry[l] = run_lane<CLS>(P, ws, i);
    });
  for (auto& t : lanes) t.join();
  for (int l = 1; l < WFA_WARP; ++l)
    if (retry[l] != retry[0]) std::abort();  // lanes disagreed: not warp-uniform
  return retry[0];
#else
  return run_lane<CLS>(P, ws, i);
#endif
}

extern "C" int64_t wfa_emu_batch(int metric, const int32_t* pen6, int compute_alignment, int span,
                                 int extension, const int32_t* free4, int hkind, const int32_t* hp3,
                                 int32_t max_steps, int format, const uint8_t* seq, int64_t seq_bytes,
                                 const int64_t* p_off, const int32_t* p_len, const int64_t* t_off,
                                 const int32_t* t_len, int64_t num_pairs, const int64_t* cigar_off,
                                 uint8_t* cigars, wfa_result_t* results, int32_t wmax,
                                 int32_t hist_scores, int64_t hist_words, int piggyback,
                                 int compat, int64_t bt_limit, int32_t bt_cap, int32_t bt_probe) {
  AlignParams P;
  std::memset(&P, 0, sizeof P);
  wfa_penalties_t u = {pen6[0], pen6[1], pen6[2], pen6[3], pen6[4], pen6[5]};
  if (set_penalties(metric, &u, P) != WFA_OK) return -1;
  P.span = span;
  P.extension = extension;
  if (free4) { P.p0 = free4[0]; P.pf = free4[1]; P.t0 = free4[2]; P.tf = free4[3]; }
  P.hkind = hkind;
  if (hp3) { P.hp0 = hp3[0]; P.hp1 = hp3[1]; P.hp2 = hp3[2]; }
  P.compute_alignment = compute_alignment;
  P.piggyback = piggyback;
  P.compat = compat;
  P.max_steps = max_steps;
  P.format = format;
  P.seq = seq;
  P.seq_bytes = seq_bytes;
  P.p_off = p_off; P.p_len = p_len; P.t_off = t_off; P.t_len = t_len;
  P.cigar_off = cigar_off;
  P.cigars = cigars;
  P.results = results;
  P.num_pairs = num_pairs;
  P.wmax = wmax < 12 ? wmax : 12;
  P.wspill = wmax;
  P.hist_scores = hist_scores;
  P.hist_words = hist_words;
  P.ring_slots = compact_ring_slots(P, metric_class(metric));
  P.desc_depth = compact_desc_depth(P, metric_class(metric));
  int32_t max_len_sum = 0;
  for (int64_t i = 0; i < num_pairs; ++i) max_len_sum = std::max(max_len_sum, p_len[i] + t_len[i]);
  if (P.piggyback && P.compute_alignment) {
    P.wmax = wmax;  // no spill ring: the ring holds offsets, pcigars and block indices
    P.wspill = 0;
    P.hist_scores = 0;
    P.hist_words = 0;
    P.bt_cap = bt_cap;
    P.bt_init_cap = max_len_sum + 8;
    P.bt_limit = bt_limit;
    P.bt_probe = bt_probe;
  }
  const int nc = metric == WFA_METRIC_GAP_AFFINE_2P ? 5 : metric == WFA_METRIC_GAP_AFFINE ? 3 : 1;
  P.dom_words = (int64_t)nc * (max_len_sum + 2 * P.scope + 5);
  int64_t retries = 0;
  int cls = metric_class(metric);
  for (int64_t i = 0; i < num_pairs; ++i) {
    bool r;
    switch (cls) {
      case kEditClass: r = run_pair<kEditClass>(P, i); break;
      case kLinearClass: r = run_pair<kLinearClass>(P, i); break;
      case kAffineClass: r = run_pair<kAffineClass>(P, i); break;
      default: r = run_pair<kAffine2pClass>(P, i); break;
    }
    if (r) { results[i].status = kStatusRetry; ++retries; }
  }
  return retries;
}

// Same dispatch as the kernel launcher: the lean instantiation without a
// heuristic, the general one with.
template <int CLS, class S>
static bool bi_lane(const AlignParams& P, const BiWorkspace& bw, int64_t i, S pat, S txt, S rpat, S rtxt) {
  if (P.hkind == WFA_HEURISTIC_NONE) return biwfa_one<CLS, S, false>(P, bw, i, pat, txt, rpat, rtxt);
  return biwfa_one<CLS, S, true>(P, bw, i, pat, txt, rpat, rtxt);
}

template <int CLS>
static bool bi_pair(const AlignParams& P, int64_t i) {
  constexpr int NC = CLS == kAffine2pClass ? 5 : CLS == kAffineClass ? 3 : 1;
  const size_t ring = (size_t)P.scope * NC;
  std::vector<WfD> d1(ring), d2(ring), d3(ring);
  const size_t ring_fr = ring + (size_t)bi_idc_rows(NC, P.e1, P.e2);
  std::vector<int32_t> v1(ring_fr * P.wmax, 0x5A5A5A5A), v2(ring_fr * P.wmax, 0x5A5A5A5A);
  std::vector<int32_t> v3(ring * P.wmax_base, 0x5A5A5A5A);
  std::vector<int4> hist((size_t)P.hist_scores, int4{0, -1, 0, 0});
  std::vector<int32_t> harena((size_t)P.hist_words, 0x5A5A5A5A);
  const int n = P.p_len[i], m = P.t_len[i];
  std::vector<uint32_t> rev((size_t)(n + m) / 4 + 16, 0);
  std::vector<uint8_t> tmp((size_t)2 * (n + m) + 16, 0);
  std::vector<BiFrame> frames(kBiMaxDepth);
  BiWorkspace bw;
  bw.fwd = Workspace{d1.data(), v1.data(), nullptr, nullptr};
  bw.rev = Workspace{d2.data(), v2.data(), nullptr, nullptr};
  bw.base = Workspace{d3.data(), v3.data(), hist.data(), harena.data()};
  bw.rev_seq = reinterpret_cast<uint8_t*>(rev.data());
  bw.cig_tmp = tmp.data();
  bw.frames = frames.data();
  auto go = [&]() -> bool {
    if (P.format == WFA_SEQ_PACKED2) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(P.seq);
      SeqPacked sp{w + P.p_off[i], n, (n + 15) >> 4};
      SeqPacked st{w + P.t_off[i], m, (m + 15) >> 4};
      uint32_t* rp = rev.data();
      uint32_t* rt = rp + ((n + 15) >> 4) + 1;
      reverse_into(sp, rp);
      reverse_into(st, rt);
      Warp::sync();
      SeqPacked rsp{rp, n, (n + 15) >> 4};
      SeqPacked rst{rt, m, (m + 15) >> 4};
      return bi_lane<CLS, SeqPacked>(P, bw, i, sp, st, rsp, rst);
    }
    SeqAscii sp{P.seq + P.p_off[i], n};
    SeqAscii st{P.seq + P.t_off[i], m};
    uint8_t* rp = bw.rev_seq;
    uint8_t* rt = rp + n + 8;
    reverse_into(sp, rp);
    reverse_into(st, rt);
    Warp::sync();
    SeqAscii rsp{rp, n};
    SeqAscii rst{rt, m};
    return bi_lane<CLS, SeqAscii>(P, bw, i, sp, st, rsp, rst);
  };
#ifdef WFA_EMU_THREADS
  EmuWarp warp;
  g_emu_warp = &warp;
  bool retry[WFA_WARP];
  std::vector<std::thread> lanes;
  for (int l = 0; l < WFA_WARP; ++l)
    lanes.emplace_back([&, l]() {
      g_emu_lane = l;
      retry[l] = go();
    });
  for (auto& t : lanes) t.join();
  for (int l = 1; l < WFA_WARP; ++l)
    if (retry[l] != retry[0]) std::abort();
  return retry[0];
#else
  return go();
#endif
}

extern "C" int64_t wfa_emu_biwfa(int metric, const int32_t* pen6, int compute_alignment, int hkind,
                                 const int32_t* hp3, int32_t max_steps, int format, const uint8_t* seq,
                                 const int64_t* p_off, const int32_t* p_len, const int64_t* t_off,
                                 const int32_t* t_len, int64_t num_pairs, const int64_t* cigar_off,
                                 uint8_t* cigars, wfa_result_t* results, int32_t wmax,
                                 int32_t hist_scores, int64_t hist_words, int32_t bi_idc) {
  AlignParams P;
  std::memset(&P, 0, sizeof P);
  wfa_penalties_t u = {pen6[0], pen6[1], pen6[2], pen6[3], pen6[4], pen6[5]};
  if (set_penalties(metric, &u, P) != WFA_OK) return -1;
  P.bi_idc = bi_idc;
  P.hkind = hkind;
  if (hp3) { P.hp0 = hp3[0]; P.hp1 = hp3[1]; P.hp2 = hp3[2]; }
  P.compute_alignment = compute_alignment;
  P.max_steps = max_steps;
  P.format = format;
  P.seq = seq;
  P.p_off = p_off; P.p_len = p_len; P.t_off = t_off; P.t_len = t_len;
  P.cigar_off = cigar_off;
  P.cigars = cigars;
  P.results = results;
  P.num_pairs = num_pairs;
  P.wmax = wmax;
  P.wmax_base = wmax < 1152 ? wmax : 1152;
  P.hist_scores = hist_scores;
  P.hist_words = hist_words;
  int64_t retries = 0;
  int cls = metric_class(metric);
  for (int64_t i = 0; i < num_pairs; ++i) {
    bool r;
    switch (cls) {
      case kEditClass: r = bi_pair<kEditClass>(P, i); break;
      case kLinearClass: r = bi_pair<kLinearClass>(P, i); break;
      case kAffineClass: r = bi_pair<kAffineClass>(P, i); break;
      default: r = bi_pair<kAffine2pClass>(P, i); break;
    }
    if (r) { results[i].status = kStatusRetry; ++retries; }
  }
  return retries;
}
