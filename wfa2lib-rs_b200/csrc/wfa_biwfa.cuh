// wfa_biwfa.cuh -- BiWFA (bidirectional WFA, O(s) memory) run by one warp per
// pair: the reference's align_biwfa / align_biwfa_score
// (src/aligner.rs:2563-3202) with its breakpoint search
// (bialign_find_breakpoint :2958-3124, src/bialign.rs:79-508), base case
// (bialign_base :3127-3202, classic backtrace) and divide-and-conquer
// recursion (bialign_recursive :2809-2950) as an explicit stack.
//
// Three PairAligner instances share the warp: forward and reverse
// (modular, score-only) and the base case (full history of every component
// for the classic affine backtrace).  The reverse aligner reads reversed
// copies of the pair's sequences made at pair start.
#pragma once

#include "wfa_align.cuh"

namespace wfab {

// src/bialign.rs:511-520
constexpr int32_t kBiFallbackMinScore = 250;
constexpr int32_t kBiFallbackMinLength = 100;
constexpr int32_t kBiRecoveryMinScore = 500;

// BI_RESTART: a breakpoint search reached its overlap scans before the I/D
// rows they read were kept (the growth phase's I/D ring ended too late); the
// search runs again with every row kept.
enum BiKind { BI_OK = 0, BI_END_REACHED, BI_UNREACHABLE, BI_MAXSTEPS, BI_UNATTAINABLE, BI_RETRY, BI_RESTART };

struct BiBreakpoint {  // BiAlignBreakpoint, src/bialign.rs:22-57
  int32_t score, sf, sr, kf, kr, of, orv, comp;
};

// A pending sub-problem of the recursion: pattern [pb, pe), text [tb, te),
// begin and end components, the score left to it.
struct BiFrame {
  int32_t pb, pe, tb, te, cb, ce, remaining;
};
// Deepest recursion kept (a pair whose stack would grow past it re-runs).
constexpr int kBiMaxDepth = 64;

// Per-pair BiWFA workspace (one lane group's).
struct BiWorkspace {
  Workspace fwd, rev, base;  // ring descriptors + cells; base also history
  uint8_t* rev_seq;          // reversed pattern then reversed text
  uint8_t* cig_tmp;          // base-case CIGAR, written backwards
  BiFrame* frames;           // the recursion's stack, kBiMaxDepth frames
};

// Diagonals per lane per pass in the BiWFA aligners (see PairAligner).
// A warp takes 4 (its wavefronts are many times its width); a team 2 (its
// width is already a large part of a wavefront, and wider unrolled passes
// add code -- instruction-fetch stalls -- and registers).
template <int LW>
constexpr int bi_unroll() { return LW > 32 ? 2 : 4; }

// GEN = false: no heuristic (the lean aligner instantiation).  LW: the lanes
// of the group aligning the pair (a warp, or a team of warps).
template <int CLS, class S, bool GEN, int LW = WFA_WARP>
struct BiDriver {
  using A = PairAligner<CLS, S, GEN, bi_unroll<LW>(), LW>;
  using G = Lanes<LW>;
  static constexpr int NC = A::NC;
  static constexpr bool AFF = A::AFF;
  static constexpr bool TWO = A::TWO;

  const AlignParams& P;
  A fwd, rev;
  // The base-case aligner is built by each base case (its state is dead
  // during the breakpoint searches, which keeps their registers free).
  Workspace base_ws;
  uint8_t* base_cg;
  BiFrame* stack;
  S pat, txt, rpat, rtxt;  // whole-pair views: forward and reversed
  int32_t n, m, lane;
  uint8_t* cg;  // output CIGAR (forward appends)
  int64_t cg_cap, cg_len;
  int32_t hkind, hp0, hp1, hp2;
  bool retry;

  WFA_D BiDriver(const AlignParams& p) : P(p), fwd(p), rev(p) {}

  static WFA_D S sub(const S& x, int begin, int len);

  WFA_D void setup(A& a, const Workspace& ws, bool modular) {
    a.ws = ws;
    a.lane = lane;
    a.scope = P.scope;
    // Ring rows as wide as this pair's wavefronts can be (trimmed inputs
    // span at most n + m + 1 diagonals, a computed range two more), so a
    // short pair's rows sit close together in the warp's slice.
    a.wmax = imin(modular ? P.wmax : P.wmax_base, n + m + 3);
    a.modular = modular;
    a.idc = false;
    a.endsfree = false;
    a.p0 = a.pf = a.t0 = a.tf = 0;
    a.hist_nc = modular ? 1 : NC;
    a.keep_null_slots = true;
    a.comp_end = CM;
    a.retry = false;
    a.hused = 0;
    a.cg = nullptr;
    a.cg_cap = 0;
  }
  WFA_D void set_heur(A& a, int mink, int maxk) {
    a.hkind = hkind; a.hp0 = hp0; a.hp1 = hp1; a.hp2 = hp2;
    if (hkind == WFA_HEURISTIC_BANDED_STATIC || hkind == WFA_HEURISTIC_BANDED_ADAPTIVE) {
      a.hp0 = mink;
      a.hp1 = maxk;
    }
  }
  WFA_D void set_seqs(A& a, bool reverse, int pb, int pe, int tb, int te) {
    a.n = pe - pb;
    a.m = te - tb;
    if (reverse) { a.pat = sub(rpat, n - pe, pe - pb); a.txt = sub(rtxt, m - te, te - tb); }
    else { a.pat = sub(pat, pb, pe - pb); a.txt = sub(txt, tb, te - tb); }
  }

  // CIGAR appends (Cigar::append_*, src/cigar.rs:79-110)
  WFA_D void append_run(uint8_t op, int64_t len) {
    if (len <= 0) return;
    if (cg_len + len > cg_cap) { retry = true; return; }
    for (int64_t i = lane; i < len; i += LW) cg[cg_len + i] = op;
    cg_len += len;
  }
  WFA_D void append_base(const A& base) {  // base.cigar [cg_begin, cg_end) forward
    int64_t len = base.cg_end - base.cg_begin;
    if (len <= 0) return;
    if (cg_len + len > cg_cap) { retry = true; return; }
    G::sync();
    for (int64_t i = lane; i < len; i += LW) cg[cg_len + i] = base.cg[base.cg_begin + i];
    cg_len += len;
    G::sync();
  }

  // bialign_overlap (src/bialign.rs:362-508) and the breakpoint scans
  // (:79-298): the first diagonal (ascending k) whose offsets meet.
  WFA_D void scan(const WfD& w0, const WfD& w1, int plen, int tlen, int s0, int s1, int go, int comp,
                  bool indel, bool forward, BiBreakpoint& bp) {
    if (s0 + s1 - go >= bp.score) return;
    // A meeting o0 + o1 >= tlen on diagonals k1 = (tlen - plen) - k0 needs
    // antidiagonals adding up to tlen + plen: skip pairs whose bounds cannot.
    if (ad_of(w0) + ad_of(w1) < tlen + plen) return;
    int lo0 = w0.lo, hi0 = w0.hi;
    int lo1i = (tlen - plen) - w1.hi, hi1i = (tlen - plen) - w1.lo;
    if (hi1i < lo0 || hi0 < lo1i) return;
    int mlo = imax(lo0, lo1i), mhi = imin(hi0, hi1i);
    int found = INT_MAX;
    for (int k0 = mlo + lane; k0 <= mhi; k0 += LW) {
      int k1 = (tlen - plen) - k0;
      int o0 = rd(w0, k0), o1 = rd(w1, k1);
      if (o0 + o1 < tlen) continue;
      if (indel) {
        int ck = forward ? k0 : k1, ch = forward ? o0 : o1;
        if (ch - ck > plen || ch > tlen) continue;
      }
      found = k0;
      break;
    }
    found = G::min(found);
    if (found == INT_MAX) return;
    int k0 = found, k1 = (tlen - plen) - k0;
    int o0 = rd(w0, k0), o1 = rd(w1, k1);
    if (forward) { bp.sf = s0; bp.sr = s1; bp.kf = k0; bp.kr = k1; bp.of = o0; bp.orv = o1; }
    else { bp.sf = s1; bp.sr = s0; bp.kf = k1; bp.kr = k0; bp.of = o1; bp.orv = o0; }
    bp.score = s0 + s1 - go;
    bp.comp = comp;
  }
  WFA_D WfD valid(A& a, int c, int s) {
    if (s < 0) return wf_none();
    WfD d = a.slot(c, s);
    return wf_is_null(d) ? wf_none() : d;
  }
  WFA_D void overlap(A& a0, A& a1, int s0, int s1, int plen, int tlen, bool forward, BiBreakpoint& bp) {
    WfD m0 = valid(a0, CM, s0);
    if (!wf_present(m0)) return;
    WfD d1_0 = AFF ? valid(a0, CD1, s0) : wf_none(), i1_0 = AFF ? valid(a0, CI1, s0) : wf_none();
    WfD d2_0 = TWO ? valid(a0, CD2, s0) : wf_none(), i2_0 = TWO ? valid(a0, CI2, s0) : wf_none();
    for (int i = 0; i < P.scope; ++i) {
      int si = s1 - i;
      if (si < 0) break;
      if (TWO && s0 + si - P.o2 < bp.score) {
        WfD w;
        if (wf_present(d2_0) && wf_present(w = valid(a1, CD2, si)))
          scan(d2_0, w, plen, tlen, s0, si, P.o2, CD2, true, forward, bp);
        if (wf_present(i2_0) && wf_present(w = valid(a1, CI2, si)))
          scan(i2_0, w, plen, tlen, s0, si, P.o2, CI2, true, forward, bp);
      }
      if (AFF && s0 + si - P.o1 < bp.score) {
        WfD w;
        if (wf_present(d1_0) && wf_present(w = valid(a1, CD1, si)))
          scan(d1_0, w, plen, tlen, s0, si, P.o1, CD1, true, forward, bp);
        if (wf_present(i1_0) && wf_present(w = valid(a1, CI1, si)))
          scan(i1_0, w, plen, tlen, s0, si, P.o1, CI1, true, forward, bp);
      }
      if (s0 + si >= bp.score) continue;
      WfD w = valid(a1, CM, si);
      if (wf_present(w)) scan(m0, w, plen, tlen, s0, si, 0, CM, false, forward, bp);
    }
  }

  // bialign_find_breakpoint, src/aligner.rs:2958-3124.  full: keep every
  // score's I/D rows from the start.  Otherwise a long search (more than
  // kBiIdcMinAd antidiagonals) stores them in the aligners' I/D rings
  // (PairAligner::idc) while the antidiagonals left to cover exceed a margin:
  // twice the growth expected over `scope` steps (a running mean) plus twice
  // the largest recent single-step growth.  The overlap scans need the last
  // `scope` scores' rows of both aligners; a search that reaches them with
  // fewer kept returns BI_RESTART.
  static constexpr int kBiIdcMinAd = 2048;
  WFA_D int find_breakpoint(int pb, int pe, int tb, int te, int cb, int ce, BiBreakpoint& bp,
                            int32_t& end_score, bool full) {
    const int plen = pe - pb, tlen = te - tb;
    set_seqs(fwd, false, pb, pe, tb, te);
    set_seqs(rev, true, pb, pe, tb, te);
    fwd.comp_end = ce;
    rev.comp_end = cb;
    const int max_ad = plen + tlen - 1;
    const bool grow_idc = !GEN && AFF && !full && P.bi_idc != 2 && (max_ad > kBiIdcMinAd || P.bi_idc == 1);
    fwd.idc = rev.idc = grow_idc;
    fwd.init_alignment_component(cb);
    rev.init_alignment_component(ce);
    if (fwd.retry || rev.retry) return BI_RETRY;
    auto quit = [&](A& a) {
      if (a.retry) return (int)BI_RETRY;
      if (a.status == WFA_STATUS_END_REACHED) { end_score = a.end_score; return (int)BI_END_REACHED; }
      return (int)BI_UNREACHABLE;
    };
    const int gap_opening = CLS == kAffineClass ? P.o1 : TWO ? imax(P.o1, P.o2) : 0;
    int sf = 0, sr = 0, fak = 0, rak = 0, ak = 0;
    // First scores whose I/D rows are kept (0: all of them); growth of
    // fak + rak per step pair: 8 x its running mean, its recent maximum.
    int keep_f = 0, keep_r = 0, mean8 = 64, gmax = 0, last_sum = 0;
    bool last_fwd = false;
    if (fwd.bi_extend(0, true, fak)) return quit(fwd);
    if (rev.bi_extend(0, true, rak)) return quit(rev);
    while (fak + rak < max_ad) {
      if (fwd.idc && P.bi_idc == 0) {
        const int g = fak + rak - last_sum;
        last_sum = fak + rak;
        mean8 += g - (mean8 >> 3);
        gmax = imax(g, gmax - (gmax >> 5));
        if (max_ad - (fak + rak) <= (P.scope * mean8) / 4 + 2 * gmax + 256) {
          fwd.idc = rev.idc = false;
          keep_f = sf + 1;
          keep_r = sr + 1;
        }
      }
      ++sf;
      fwd.bi_compute(sf);
      if (fwd.retry) return BI_RETRY;
      bool done = fwd.bi_extend(sf, true, ak);
      fak = imax(fak, ak);
      last_fwd = true;
      if (done) return quit(fwd);
      if (fak + rak >= max_ad) break;
      ++sr;
      rev.bi_compute(sr);
      if (rev.retry) return BI_RETRY;
      done = rev.bi_extend(sr, true, ak);
      rak = imax(rak, ak);
      last_fwd = false;
      if (done) return quit(rev);
      if (sf + sr >= P.max_steps) return BI_MAXSTEPS;
    }
    const int scope = P.scope;
    if (grow_idc && (fwd.idc || keep_f > imax(0, sf - (scope - 1)) || keep_r > imax(0, sr - (scope - 1))))
      return BI_RESTART;
    fwd.idc = rev.idc = false;
    for (;;) {
      if (last_fwd) {
        int min_sr = sr > scope - 1 ? sr - (scope - 1) : 0;
        if (sf + min_sr - gap_opening >= bp.score) break;
        overlap(fwd, rev, sf, sr, plen, tlen, true, bp);
        ++sr;
        rev.bi_compute(sr);
        if (rev.retry) return BI_RETRY;
        if (rev.bi_extend(sr, false, ak)) return quit(rev);
      }
      int min_sf = sf > scope - 1 ? sf - (scope - 1) : 0;
      if (min_sf + sr - gap_opening >= bp.score) break;
      overlap(rev, fwd, sr, sf, plen, tlen, false, bp);
      ++sf;
      fwd.bi_compute(sf);
      if (fwd.retry) return BI_RETRY;
      if (fwd.bi_extend(sf, false, ak)) return quit(fwd);
      if (sf + sr >= P.max_steps) return BI_MAXSTEPS;
      last_fwd = true;
    }
    return BI_OK;
  }
  WFA_D int find_breakpoint(int pb, int pe, int tb, int te, int cb, int ce, BiBreakpoint& bp,
                            int32_t& end_score) {
    int st = find_breakpoint(pb, pe, tb, te, cb, ce, bp, end_score, false);
    if (st == BI_RESTART) st = find_breakpoint(pb, pe, tb, te, cb, ce, bp, end_score, true);
    return st;
  }

  // bialign_base, src/aligner.rs:3127-3202
  WFA_D int base_case(int pb, int pe, int tb, int te, int cb, int ce, int32_t& result) {
    A base(P);
    setup(base, base_ws, false);
    base.cg = base_cg;
    set_heur(base, hp0 - (tb - pb), hp1 - (tb - pb));
    set_seqs(base, false, pb, pe, tb, te);
    base.cap = imax(base.dims_num(1000, 1000), base.dims_num(base.n, base.m));
    base.comp_end = ce;
    base.cg_cap = 2 * ((int64_t)base.n + base.m) + 1;
    base.init_alignment_component(cb);
    if (base.retry) return BI_RETRY;
    int score = 0, ak;
    for (;;) {
      bool done = base.bi_extend(score, false, ak);
      base.hist_commit(score);
      if (base.retry) return BI_RETRY;
      if (done) break;
      ++score;
      if (!base.has_slot(score)) { base.status = WFA_STATUS_MAX_STEPS_REACHED; break; }
      base.bi_compute(score);
      if (base.retry) return BI_RETRY;
      if (score >= INT_MAX) { base.status = WFA_STATUS_MAX_STEPS_REACHED; break; }
    }
    int st = BI_OK;
    base.cg_begin = 0;
    base.cg_end = 0;
    if (base.status == WFA_STATUS_END_REACHED) {
      base.backtrace_components(score, base.end_k, base.end_off, ce);
      result = score;
    } else if (base.status == WFA_STATUS_END_UNREACHABLE && base.end_off != kOffsetNull) {
      // C: from component_end at the best cell's score; Corrected: from M
      // (the best cell is an M cell), src/aligner.rs:3181-3192.
      if (P.compat == WFA_COMPAT_CORRECTED) {
        base.backtrace_components(base.end_score, base.end_k, base.end_off, CM);
      } else {
        int from = base.end_score >= 0 ? base.end_score : score;
        base.backtrace_components(from, base.end_k, base.end_off, ce);
      }
      base.maxtrim_cigar();
      st = BI_UNATTAINABLE;
    } else {
      base.cg_begin = 0;
      base.cg_end = 0;
      st = BI_UNATTAINABLE;
    }
    if (base.status == WFA_STATUS_OOM) return BI_RETRY;
    append_base(base);
    return st;
  }

  // bialign_recursive, src/aligner.rs:2809-2950, with an explicit stack in
  // the group's workspace (shared memory in the kernel): lane 0 pushes, and
  // a sync separates every push from the reads of the frames it writes.
  WFA_D void push(int& top, const BiFrame& f) {
    if (lane == 0) stack[top] = f;
    ++top;
  }
  WFA_D int recursive(int32_t& result) {
    int top = 0;
    push(top, BiFrame{0, n, 0, m, CM, CM, imax(n, m) <= kBiFallbackMinLength ? 0 : INT_MAX});
    bool first = true;
    int32_t top_result = 0;
    while (top > 0) {
      G::sync();
      const BiFrame f = stack[--top];
      const int plen = f.pe - f.pb, tlen = f.te - f.tb;
      int32_t r = 0;
      if (tlen == 0) {
        append_run('D', plen);
        if (retry) return BI_RETRY;
        if (first) top_result = 0;
        first = false;
        continue;
      }
      if (plen == 0) {
        append_run('I', tlen);
        if (retry) return BI_RETRY;
        if (first) top_result = 0;
        first = false;
        continue;
      }
      if (f.remaining <= kBiFallbackMinScore) {
        int st = base_case(f.pb, f.pe, f.tb, f.te, f.cb, f.ce, r);
        if (st != BI_OK) return st;
        if (first) top_result = r;
        first = false;
        continue;
      }
      int shift = f.tb - f.pb, diag = tlen - plen;
      set_heur(fwd, hp0 - shift, hp1 - shift);
      set_heur(rev, diag - (hp1 - shift), diag - (hp0 - shift));
      BiBreakpoint bp;
      bp.score = INT_MAX; bp.sf = bp.sr = bp.kf = bp.kr = bp.of = bp.orv = 0; bp.comp = CM;
      int32_t es = 0;
      int st = find_breakpoint(f.pb, f.pe, f.tb, f.te, f.cb, f.ce, bp, es);
      if (st == BI_RETRY) return BI_RETRY;
      if (st == BI_END_REACHED) {
        if (es <= kBiRecoveryMinScore) {
          st = base_case(f.pb, f.pe, f.tb, f.te, f.cb, f.ce, r);
          if (st != BI_OK) return st;
          if (first) top_result = r;
          first = false;
          continue;
        }
        return BI_UNREACHABLE;
      }
      if (st != BI_OK) return st;
      if (first) top_result = bp.score;
      first = false;
      if (top + 2 > kBiMaxDepth) return BI_RETRY;
      const int bph = bp.of, bpv = bp.of - bp.kf;
      // Right half is processed after the left one (pushed first).
      G::sync();  // every lane has read the frame popped last
      push(top, BiFrame{f.pb + bpv, f.pe, f.tb + bph, f.te, bp.comp, f.ce, bp.sr});
      push(top, BiFrame{f.pb, f.pb + bpv, f.tb, f.tb + bph, f.cb, bp.comp, bp.sf});
    }
    result = top_result;
    return BI_OK;
  }
};

template <int CLS, class S, bool GEN, int LW>
WFA_D S BiDriver<CLS, S, GEN, LW>::sub(const S& x, int begin, int len) {
  S v = x;
  if constexpr (S::UNITS == 16) {
    v.off = x.off + begin;
  } else {
    v.p = x.p + begin;
  }
  v.len = len;
  return v;
}

// align_biwfa (src/aligner.rs:2563-2644) or align_biwfa_score (:2650-2698)
// of pair `pair`; writes its result.  Returns true to retry with more scratch.
template <int CLS, class S, bool GEN, int LW = WFA_WARP>
WFA_D bool biwfa_one(const AlignParams& P, const BiWorkspace& bw, int64_t pair, S pat, S txt,
                     S rpat, S rtxt) {
  using D_t = BiDriver<CLS, S, GEN, LW>;
  D_t D(P);
  D.lane = Lanes<LW>::lane();
  D.n = P.p_len[pair];
  D.m = P.t_len[pair];
  D.pat = pat; D.txt = txt; D.rpat = rpat; D.rtxt = rtxt;
  D.hkind = P.hkind; D.hp0 = P.hp0; D.hp1 = P.hp1; D.hp2 = P.hp2;
  D.retry = false;
  D.setup(D.fwd, bw.fwd, true);
  D.setup(D.rev, bw.rev, true);
  D.base_ws = bw.base;
  D.base_cg = bw.cig_tmp;
  D.stack = bw.frames;
  const int n = D.n, m = D.m;
  int32_t score = 0, status;
  D.cg = nullptr;
  D.cg_cap = 0;
  D.cg_len = 0;
  int32_t cig_score = INT_MIN, ev = -1, eh = -1;
  if (!P.compute_alignment) {
    // align_biwfa_score: the first breakpoint's score, or the end's.
    D.set_heur(D.fwd, P.hp0, P.hp1);
    D.set_heur(D.rev, (m - n) - P.hp1, (m - n) - P.hp0);
    BiBreakpoint bp;
    bp.score = INT_MAX; bp.sf = bp.sr = bp.kf = bp.kr = bp.of = bp.orv = 0; bp.comp = CM;
    int32_t es = 0;
    int st = D.find_breakpoint(0, n, 0, m, CM, CM, bp, es);
    if (st == BI_RETRY) return true;
    score = st == BI_OK ? bp.score : st == BI_END_REACHED ? es : 0;
    status = (st == BI_OK || st == BI_END_REACHED) ? WFA_STATUS_COMPLETED
             : st == BI_MAXSTEPS ? WFA_STATUS_MAX_STEPS_REACHED : WFA_STATUS_END_UNREACHABLE;
  } else {
    D.cg = P.cigars + P.cigar_off[pair];
    D.cg_cap = 2 * ((int64_t)n + m) + 1;
    int32_t result = 0;
    int st = D.recursive(result);
    if (st == BI_RETRY || D.retry) return true;
    if (st == BI_OK) {
      bool heur = P.hkind != WFA_HEURISTIC_NONE && D.cg_len > 0;
      if (n == 0 || m == 0 || heur) {
        typename D_t::A sc(P);
        D.setup(sc, bw.base, false);
        sc.cg = D.cg;
        score = sc.cigar_wfa_score(0, D.cg_len, n, m);
      } else {
        score = result;
      }
      cig_score = score;
      ev = n;
      eh = m;
      status = WFA_STATUS_COMPLETED;
    } else {
      status = st == BI_MAXSTEPS ? WFA_STATUS_MAX_STEPS_REACHED : WFA_STATUS_END_UNREACHABLE;
      score = 0;
    }
  }
  Lanes<LW>::sync();
  if (D.lane == 0) {
    wfa_result_t r;
    r.score = score;
    r.status = status;
    r.cigar_begin = 0;
    r.cigar_length = (int32_t)D.cg_len;
    r.cigar_score = cig_score;
    r.end_v = ev;
    r.end_h = eh;
    r.end_score = 0;  // the BiWFA aligner's own end position is never set
    r.end_k = 0;
    r.end_offset = 0;
    P.results[pair] = r;
  }
  return false;
}

// Reversed copies of a pair's sequences for the reverse aligner.
template <int LW = WFA_WARP>
WFA_D void reverse_into(const SeqPacked& s, uint32_t* out) {
  const int nw = (s.len + 15) >> 4;
  for (int j = Lanes<LW>::lane(); j < nw; j += LW) {
    uint32_t x = s.fetch(s.len - 16 * (j + 1));
    // reverse the order of the sixteen 2-bit codes
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    x = (x >> 16) | (x << 16);
    out[j] = x;
  }
}
template <int LW = WFA_WARP>
WFA_D void reverse_into(const SeqAscii& s, uint8_t* out) {
  for (int i = Lanes<LW>::lane(); i < s.len; i += LW) out[i] = s.p[s.len - 1 - i];
}

}  // namespace wfab
