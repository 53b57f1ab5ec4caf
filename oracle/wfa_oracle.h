/*
 * wfa_oracle.h -- C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement of the
 * wfa2lib-rs CPU alignment path (src/aligner.rs and the modules it drives).
 * It is the checker for the CUDA path and the timed CPU baseline ("port").
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it; the product library never links or calls it.
 *
 * Parity is pinned by the golden vectors under tests/golden/ (extracted from
 * the reference's own tests and data files by tests/golden/make_golden.py).
 */
#ifndef WFA_ORACLE_H
#define WFA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Metric ids follow DistanceMetric (src/penalties.rs:12-23). */
enum { WFO_INDEL = 0, WFO_EDIT = 1, WFO_LINEAR = 2, WFO_AFFINE = 3, WFO_AFFINE2P = 4 };
/* AlignStatus (src/aligner.rs:120-135). */
enum {
  WFO_STATUS_OK = 0, WFO_STATUS_END_REACHED = 1, WFO_STATUS_END_UNREACHABLE = 2,
  WFO_STATUS_MAX_STEPS = 3, WFO_STATUS_OOM = 4, WFO_STATUS_COMPLETED = 5, WFO_STATUS_PARTIAL = 6
};
/* HeuristicStrategy (src/heuristic.rs:14-58). */
enum {
  WFO_H_NONE = 0, WFO_H_WFADAPTIVE = 1, WFO_H_XDROP = 2, WFO_H_ZDROP = 3,
  WFO_H_BANDED_STATIC = 4, WFO_H_BANDED_ADAPTIVE = 5
};
/* MemoryMode (src/aligner.rs:43-51). */
enum { WFO_MEM_HIGH = 0, WFO_MEM_MED = 1, WFO_MEM_LOW = 2 };

/* pen[6] = user penalties: linear (match, mismatch, indel), affine
 * (match, mismatch, open, extend), affine2p (match, mismatch, o1, e1, o2, e2).
 * Returns NULL when the penalties are invalid (the reference panics). */
void* wfo_create(int metric, const int32_t* pen);
void wfo_destroy(void* h);
void wfo_set_alignment_scope(void* h, int compute_alignment);
void wfo_set_memory_mode(void* h, int mode);
void wfo_set_compat(void* h, int compat);  // 0 C, 1 Corrected (src/aligner.rs:53-94)
/* Med/low with an alignment: 1 (default) runs the reference's piggyback
 * path as it is (per-cell packed CIGARs and backtrace-buffer blocks,
 * src/compute/piggyback.rs, src/bt_buffer.rs); 0 re-makes the kernels' picks
 * from the kept offsets after the end cell is found (the design the GPU
 * library uses).  Both give the same results. */
void wfo_set_piggyback_literal(void* h, int on);
void wfo_set_heuristic(void* h, int kind, int32_t p0, int32_t p1, int32_t p2);
void wfo_set_max_alignment_steps(void* h, int32_t steps);
void wfo_set_alignment_free_ends(void* h, int32_t p0, int32_t pf, int32_t t0, int32_t tf);
void wfo_set_alignment_extension(void* h);
void wfo_set_alignment_end_to_end(void* h);

int32_t wfo_align_end2end(void* h, const char* p, int32_t n, const char* t, int32_t m);
int32_t wfo_align_endsfree(void* h, const char* p, int32_t n, const char* t, int32_t m);
int32_t wfo_align_biwfa(void* h, const char* p, int32_t n, const char* t, int32_t m);
int32_t wfo_align_biwfa_score(void* h, const char* p, int32_t n, const char* t, int32_t m);
int32_t wfo_align_packed2bits(void* h, const uint8_t* p, int32_t n, const uint8_t* t, int32_t m);

int wfo_status(void* h);
/* CIGAR of the last alignment: copies at most cap ops, returns the length. */
int32_t wfo_cigar(void* h, char* ops, int32_t cap, int32_t* score, int32_t* end_v, int32_t* end_h);
void wfo_end_pos(void* h, int32_t* score, int32_t* k, int32_t* offset);
/* Algorithmic work counters of the last alignment: cells computed (sum of
 * hi-lo+1 over set_limits), bases compared by extend, CIGAR ops. */
void wfo_counters(void* h, int64_t* cells, int64_t* bases, int64_t* ops);

/* align_benchmark output line for one pair ("score\tCIGAR"), following
 * src/bin/align_benchmark.rs:593-672.  span: 0 global, 1 extension,
 * 2 ends-free with free[4] (already resolved to counts).  Returns the line
 * length or -1 if the driver would exit with an error. */
int32_t wfo_cli_line(void* h, int span, const int32_t* free4, int biwfa, int score_only,
                     const char* p, int32_t n, const char* t, int32_t m, char* out, int32_t cap);

/* Multi-threaded batch (CPU baseline): pairs i in [0,count) at
 * seq + p_off[i] (length p_len[i]) and seq + t_off[i] (t_len[i]); mode 0
 * end2end, 1 endsfree, 2 biwfa.  Returns wall seconds of the align calls
 * (max over threads).  scores/status/cigar_hash may be NULL; work3, if
 * not NULL, receives the sums over the batch of the wfo_counters figures
 * (cells computed, bases compared, CIGAR ops). */
double wfo_batch(int metric, const int32_t* pen, int compute_alignment, int mode,
                 int heuristic_kind, const int32_t* hparams, const int32_t* free4,
                 const char* seq, const int64_t* p_off, const int32_t* p_len,
                 const int64_t* t_off, const int32_t* t_len, int64_t count, int threads,
                 int32_t* scores, int32_t* status, int64_t* cigar_hash, int64_t* work3);

/* FNV-1a 64-bit hash of ops[begin[i] .. begin[i] + len[i]) for every i (the
 * same hash wfo_batch reports per CIGAR), so a CIGAR buffer produced
 * elsewhere compares against the oracle's without copying CIGARs around. */
void wfo_hash_ops(const uint8_t* ops, const int64_t* begin, const int32_t* len, int64_t count,
                  int threads, int64_t* out);

#ifdef __cplusplus
}
#endif
#endif
