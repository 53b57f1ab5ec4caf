/*
 * wfa_b200.h -- C ABI of the B200 wavefront-alignment library.
 *
 * The entry points replace the public aligner API of wfa2lib-rs
 * (src/aligner.rs, `WavefrontAligner<N>`), one C function per Rust method,
 * so that a Rust (or any FFI) caller binds them 1:1; INTEGRATION.md shows the
 * binding.  Everything is plain pointers, sizes and integer codes.  Errors are
 * negative return codes (never an abort): where the reference panics on
 * invalid penalties (src/penalties.rs:157-167,198-209,253-265) the C ABI
 * returns WFA_ERR_PENALTIES.
 *
 * Threading: a handle is used by one host thread at a time (the reference's
 * aligner is Send, not Sync).  Different handles may run concurrently.
 *
 * Results are bit-identical to the reference's CPU path (score, CIGAR,
 * tie-breaks, statuses) for every pair; each pair of a batch is aligned as a
 * freshly created reference aligner with the handle's configuration would
 * align it.
 */
#ifndef WFA_B200_H
#define WFA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define WFA_API __attribute__((visibility("default")))
#else
#define WFA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums (values match the reference's enum order) ------------------ */

/* DistanceMetric, src/penalties.rs:12-23 */
typedef enum {
  WFA_METRIC_INDEL = 0,
  WFA_METRIC_EDIT = 1,
  WFA_METRIC_GAP_LINEAR = 2,
  WFA_METRIC_GAP_AFFINE = 3,
  WFA_METRIC_GAP_AFFINE_2P = 4
} wfa_metric_t;

/* AlignStatus, src/aligner.rs:120-135 */
typedef enum {
  WFA_STATUS_OK = 0,
  WFA_STATUS_END_REACHED = 1,
  WFA_STATUS_END_UNREACHABLE = 2,
  WFA_STATUS_MAX_STEPS_REACHED = 3,
  WFA_STATUS_OOM = 4,
  WFA_STATUS_COMPLETED = 5,
  WFA_STATUS_PARTIAL = 6
} wfa_status_t;

/* AlignmentScope, src/aligner.rs:26-31 */
typedef enum { WFA_SCOPE_SCORE = 0, WFA_SCOPE_ALIGNMENT = 1 } wfa_scope_t;

/* MemoryMode, src/aligner.rs:43-51 (BiWFA / "ultralow" is wfa_align_biwfa) */
typedef enum { WFA_MEMORY_HIGH = 0, WFA_MEMORY_MED = 1, WFA_MEMORY_LOW = 2 } wfa_memory_t;

/* Compat, src/aligner.rs:88-94 */
typedef enum { WFA_COMPAT_C = 0, WFA_COMPAT_CORRECTED = 1 } wfa_compat_t;

/* HeuristicStrategy, src/heuristic.rs:14-58 */
typedef enum {
  WFA_HEURISTIC_NONE = 0,
  WFA_HEURISTIC_WFADAPTIVE = 1,   /* p0 min_wavefront_length, p1 max_distance_threshold, p2 steps */
  WFA_HEURISTIC_XDROP = 2,        /* p0 xdrop, p1 steps_between_cutoffs */
  WFA_HEURISTIC_ZDROP = 3,        /* p0 zdrop, p1 steps_between_cutoffs */
  WFA_HEURISTIC_BANDED_STATIC = 4,   /* p0 min_k, p1 max_k */
  WFA_HEURISTIC_BANDED_ADAPTIVE = 5  /* p0 min_k, p1 max_k, p2 steps */
} wfa_heuristic_kind_t;

/* Error codes (negative). */
enum {
  WFA_OK = 0,
  WFA_ERR_PENALTIES = -1,   /* invalid penalties (the reference panics) */
  WFA_ERR_ARGUMENT = -2,    /* NULL handle / bad size / bad enum */
  WFA_ERR_UNSUPPORTED = -3, /* configuration this build does not run on the GPU */
  WFA_ERR_CUDA = -4,        /* CUDA runtime error (see wfa_last_error_string) */
  WFA_ERR_NO_DEVICE = -5,   /* no CUDA device */
  WFA_ERR_OOM = -6,         /* device memory exhausted */
  WFA_ERR_BUSY = -7         /* a resident stream's request ring is full: poll, then submit again */
};

/* ---- penalties ---------------------------------------------------------- */

/* User penalties, as the reference's LinearPenalties / AffinePenalties /
 * Affine2pPenalties (src/penalties.rs:26-65).  Gap-linear puts `indel` in
 * gap_opening1.  Unused fields are ignored. */
typedef struct {
  int32_t match;
  int32_t mismatch;
  int32_t gap_opening1;
  int32_t gap_extension1;
  int32_t gap_opening2;
  int32_t gap_extension2;
} wfa_penalties_t;

/* Replaces the validation asserts of WavefrontPenalties::new_linear/
 * new_affine/new_affine2p (src/penalties.rs:157-296).  WFA_OK or
 * WFA_ERR_PENALTIES. */
WFA_API int wfa_penalties_check(wfa_metric_t metric, const wfa_penalties_t* penalties);

/* ---- aligner handle ----------------------------------------------------- */

typedef struct wfa_aligner wfa_aligner_t;

/* WavefrontAligner::new (src/aligner.rs:409).  `device` is the CUDA device
 * ordinal.  Returns NULL and sets *err (if err != NULL) on failure. */
WFA_API wfa_aligner_t* wfa_aligner_create(wfa_metric_t metric, const wfa_penalties_t* penalties,
                                  int device, int* err);
WFA_API void wfa_aligner_destroy(wfa_aligner_t* h);

/* Builder setters, src/aligner.rs:462-613.  Return WFA_OK or an error.
 * Med/low memory with an alignment gives the reference's med/low CIGARs (its
 * piggyback backtrace); the device keeps every component's history for it,
 * so wfa_set_max_memory_compact (the reference's backtrace-buffer compaction
 * limit) is accepted and has no effect on results or on device memory. */
WFA_API int wfa_set_memory_mode(wfa_aligner_t* h, wfa_memory_t mode);               /* :462 */
WFA_API int wfa_set_max_memory_compact(wfa_aligner_t* h, uint64_t bytes);           /* :469 */
WFA_API int wfa_set_max_alignment_steps(wfa_aligner_t* h, int32_t max_steps);       /* :533 */
WFA_API int wfa_set_alignment_scope(wfa_aligner_t* h, wfa_scope_t scope);           /* :542 */
WFA_API int wfa_set_alignment_free_ends(wfa_aligner_t* h, int32_t pattern_begin_free,
                                int32_t pattern_end_free, int32_t text_begin_free,
                                int32_t text_end_free);                      /* :563 */
WFA_API int wfa_set_alignment_extension(wfa_aligner_t* h);                          /* :582 */
WFA_API int wfa_set_alignment_end_to_end(wfa_aligner_t* h);                         /* :595 */
WFA_API int wfa_set_compat(wfa_aligner_t* h, wfa_compat_t compat);                  /* :606 */
WFA_API int wfa_set_heuristic(wfa_aligner_t* h, wfa_heuristic_kind_t kind, int32_t p0, int32_t p1,
                      int32_t p2);                                          /* :611 */

/* ---- plain per-call aligners (host buffers) -------------------------------
 * Each returns the alignment score (what the Rust method returns) or, when
 * the call itself fails, a negative WFA_ERR_* code with wfa_status() ==
 * WFA_STATUS_OOM and wfa_last_error() set.  Sequences are ASCII bytes. */
WFA_API int32_t wfa_align_end2end(wfa_aligner_t* h, const uint8_t* pattern, int32_t pattern_length,
                          const uint8_t* text, int32_t text_length);            /* :620 */
WFA_API int32_t wfa_align_endsfree(wfa_aligner_t* h, const uint8_t* pattern, int32_t pattern_length,
                           const uint8_t* text, int32_t text_length);           /* :707 */
WFA_API int32_t wfa_align_biwfa(wfa_aligner_t* h, const uint8_t* pattern, int32_t pattern_length,
                        const uint8_t* text, int32_t text_length);              /* :2563 */
WFA_API int32_t wfa_align_biwfa_score(wfa_aligner_t* h, const uint8_t* pattern,
                              int32_t pattern_length, const uint8_t* text,
                              int32_t text_length);                              /* :2650 */
/* 2-bit packed input, 4 bases per byte LSB-first (A0 C1 G2 T3), as
 * align_packed2bits (src/aligner.rs:2755, src/sequences.rs:55-74). */
WFA_API int32_t wfa_align_packed2bits(wfa_aligner_t* h, const uint8_t* pattern, int32_t pattern_length,
                              const uint8_t* text, int32_t text_length);
/* align_lambda (src/aligner.rs:2743) needs a host callback per base
 * comparison; it cannot run on the device: always WFA_ERR_UNSUPPORTED. */
WFA_API int32_t wfa_align_lambda(wfa_aligner_t* h, int (*match_fn)(int32_t, int32_t, void*), void* ctx,
                         int32_t pattern_length, int32_t text_length);

/* Accessors: status() (:834), cigar() (:839), alignment_end_pos (pub field).
 * The CIGAR pointer stays valid until the next call on the handle. */
WFA_API wfa_status_t wfa_status(const wfa_aligner_t* h);
WFA_API int wfa_cigar(const wfa_aligner_t* h, const uint8_t** ops, int32_t* length, int32_t* score,
              int32_t* end_v, int32_t* end_h);
WFA_API int wfa_alignment_end_pos(const wfa_aligner_t* h, int32_t* score, int32_t* k, int32_t* offset);
WFA_API int wfa_last_error(const wfa_aligner_t* h);
WFA_API const char* wfa_last_error_string(const wfa_aligner_t* h);

/* ---- batched form ---------------------------------------------------------
 * Many pairs in one launch of the persistent kernel.  Sequences live in one
 * buffer: pattern i is seq[p_off[i] .. p_off[i]+p_len[i]) and text i likewise
 * (ASCII: byte offsets; WFA_SEQ_PACKED2: 32-bit-word offsets into a buffer of
 * 2-bit codes, 16 bases per word LSB-first, every sequence word-aligned).
 * Per pair the result goes to results[i]; CIGAR ops ('M','X','I','D') of pair
 * i are written inside its slot cigars[cigar_off[i] .. + cigar_cap(i)) with
 * cigar_cap(i) = 2*(p_len+t_len)+1 (wfa_batch_align_device: results[i].
 * cigar_begin is relative to that slot; wfa_batch_align: the CIGARs are
 * packed densely in input order and cigar_begin is the offset into `cigars`). */
typedef enum { WFA_SEQ_ASCII = 0, WFA_SEQ_PACKED2 = 1 } wfa_seq_format_t;
/* Which reference call each pair follows: align_end2end, align_endsfree, or
 * BiWFA (align_biwfa in alignment scope, align_biwfa_score in score scope). */
typedef enum { WFA_SPAN_END2END = 0, WFA_SPAN_ENDSFREE = 1, WFA_SPAN_BIWFA = 2 } wfa_span_mode_t;

typedef struct {
  int32_t score;        /* what align_* returns */
  int32_t status;       /* wfa_status_t */
  int32_t cigar_begin;  /* first op, relative to the pair's slot */
  int32_t cigar_length; /* 0 in score-only mode */
  int32_t cigar_score;  /* Cigar::score */
  int32_t end_v;        /* Cigar::end_v */
  int32_t end_h;        /* Cigar::end_h */
  int32_t end_score;    /* alignment_end_pos.score */
  int32_t end_k;        /* alignment_end_pos.k */
  int32_t end_offset;   /* alignment_end_pos.offset */
} wfa_result_t;

typedef struct {
  int32_t format;           /* wfa_seq_format_t */
  int32_t span;             /* wfa_span_mode_t: align_end2end or align_endsfree semantics */
  int64_t num_pairs;
  const void* seq;          /* sequence buffer */
  int64_t seq_bytes;        /* its size in bytes */
  const int64_t* p_off;
  const int32_t* p_len;
  const int64_t* t_off;
  const int32_t* t_len;
  const int64_t* cigar_off; /* NULL in score-only mode */
  int64_t cigar_bytes;      /* size of the CIGAR buffer */
} wfa_batch_t;

/* Host-buffer batch: copies inputs to the device, aligns every pair, copies
 * results (and CIGARs) back.  cigars may be NULL in score-only mode.  Blocks
 * until done.  Returns WFA_OK or an error code. */
WFA_API int wfa_batch_align(wfa_aligner_t* h, const wfa_batch_t* batch, wfa_result_t* results,
                    uint8_t* cigars);

/* Device-buffer batch: every pointer of `batch`, `results` and `cigars` is
 * device memory; the work runs on `stream` (a cudaStream_t, 0 for the
 * handle's own stream).  The call synchronises that stream to read the
 * longest pair and the number of pairs to re-run with more scratch, so the
 * results are complete when it returns.  Scratch memory is owned by the
 * handle and reused across calls. */
WFA_API int wfa_batch_align_device(wfa_aligner_t* h, const wfa_batch_t* batch, wfa_result_t* results,
                           uint8_t* cigars, void* stream);

/* Asynchronous host-buffer batch: queues the batch of wfa_batch_align and
 * returns a ticket (>= 0) at once.  The batch's arrays, `results` and
 * `cigars` are the caller's and must stay valid and untouched until the
 * ticket completes.  A handle's batches run one after another, in
 * submission order, on a worker thread the first submit starts; while
 * tickets are outstanding, use no other call of the handle.
 * wfa_batch_poll returns 1 (and the batch's return code in *status) once the
 * ticket is done, 0 before; wfa_batch_wait blocks until then and returns that
 * code.  A completed ticket is reported once. */
WFA_API int64_t wfa_batch_submit(wfa_aligner_t* h, const wfa_batch_t* batch, wfa_result_t* results,
                                 uint8_t* cigars);
WFA_API int wfa_batch_poll(wfa_aligner_t* h, int64_t ticket, int* status);
WFA_API int wfa_batch_wait(wfa_aligner_t* h, int64_t ticket);

/* ---- device-buffer batch that allocates nothing -----------------------------
 * No counterpart in the reference: an addition of this library.
 *
 * wfa_batch_align_device grows a scratch buffer with cudaMalloc/cudaFree as
 * batches need it.  Some callers cannot allow that: a plug-in inside a host
 * program whose own allocator has already reserved the device memory (a
 * framework's caching allocator, a server's arena) can see cudaMalloc fail
 * although the caller has room to spare, and cudaFree waits for the whole
 * device, stalling every other stream of the program.  This entry point
 * takes the same arguments and gives the same results, but its scratch is
 * one fixed device array of WFA_NOALLOC_SCRATCH_BYTES that the library holds
 * on each device where it has been used, until the process exits; it calls
 * no allocation routine.
 *
 * - The first call on a device looks up the array's device address (again
 *   after the device's context was re-created, e.g. by cudaDeviceReset);
 *   make that first call before any stream capture.
 * - Limits: the longest pair of the batch must have p_len + t_len <=
 *   WFA_NOALLOC_MAX_LEN_SUM, else WFA_ERR_ARGUMENT; an alignment that needs
 *   more scratch than a quarter of the array fails with WFA_ERR_OOM (use
 *   wfa_batch_align_device for it).  Spans end-to-end and ends-free; BiWFA
 *   gives WFA_ERR_UNSUPPORTED.
 * - Every call on a device shares the one array, which keeps what the last
 *   call left in it (each call zeroes the counters it needs first).  Calls
 *   whose work overlaps on the same device (two streams, two handles, two
 *   threads) race on it: serialise them.
 * - Like wfa_batch_align_device it synchronises `stream` to read the longest
 *   pair and the number of pairs to re-run. */
#define WFA_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define WFA_NOALLOC_MAX_LEN_SUM 4096
WFA_API int wfa_batch_align_device_noalloc(wfa_aligner_t* h, const wfa_batch_t* batch,
                                           wfa_result_t* results, uint8_t* cigars, void* stream);

/* ---- serving: continuous batching of single requests ------------------------
 * No counterpart in the reference (its aligner is one pair per call): a
 * request loop in front of the batched kernels.  Requests are submitted one
 * at a time from any thread and sorted into three lanes: short (n + m up to
 * `short_max_len`), long high-memory and BiWFA.  Each lane has its own
 * workers, each worker its own aligner handle, stream and buffers, so
 * several batches are on the GPU at once and a short request never waits
 * behind a long batch.  A worker that frees up takes every waiting request
 * of its lane that fits into its next batch, so a request arriving while
 * others are on the GPU joins the next free batch instead of waiting for
 * the whole queue.
 *
 * Admission is by predicted wavefront memory: a request's high-memory
 * footprint is taken as (n + m)^2 / 4 bytes (M history of O(s^2) cells with
 * s about (n + m) / 4) and its BiWFA footprint as O(n + m).  A request whose
 * high-memory estimate is above `biwfa_above_bytes` runs in BiWFA; a batch
 * takes requests in arrival order while the sum of their estimates stays
 * within `max_batch_bytes` (a request larger than that alone gets a batch
 * of its own).  The mode of a request depends only on its lengths and the
 * configuration, never on the load, so a request gets the same result alone
 * or in a mix (the result of align_end2end, or of align_biwfa, with the
 * server's metric, penalties and scope). */
typedef struct {
  int32_t metric;               /* wfa_metric_t */
  wfa_penalties_t penalties;
  int32_t device;
  int32_t score_only;           /* 1: alignment scope score only */
  int32_t workers;              /* long high-memory lane workers (default 2) */
  int32_t max_batch_pairs;      /* per batch (default 65536) */
  int64_t max_batch_bytes;      /* predicted wavefront bytes per batch (default 4 GiB) */
  int64_t biwfa_above_bytes;    /* BiWFA above this estimate (default 256 MiB) */
  int32_t short_workers;        /* short lane workers (default 2) */
  int32_t biwfa_workers;        /* BiWFA lane workers (default 2) */
  int32_t short_max_len;        /* n + m of the short lane (default 1024) */
  int32_t resident;             /* 1: the short lane is a resident stream (wfa_stream_*; n + m of the
                                   short lane at most 2048).  Measured: the long and BiWFA lanes'
                                   batches then wait until the resident kernel has ended (a second
                                   after the last request); use it for short-read traffic. */
} wfa_server_config_t;

typedef struct wfa_server wfa_server_t;

typedef struct {
  int64_t id;            /* as returned by wfa_server_submit */
  int32_t score;         /* what align_end2end / align_biwfa returns */
  int32_t status;        /* wfa_status_t, or the batch's error code (< 0) */
  int32_t cigar_length;  /* ops at cigars[cigar_offset] of the poll buffer */
  int32_t cigar_score;
  int32_t end_v, end_h;
  int32_t mode;          /* 0 high memory (end-to-end), 1 BiWFA */
  int32_t pad;
  int64_t cigar_offset;
  int64_t latency_ns;    /* submit to result ready */
} wfa_served_t;

/* Starts the workers; NULL on error (*err set). */
WFA_API wfa_server_t* wfa_server_start(const wfa_server_config_t* config, int* err);
/* Queues one pair (copied); returns its id (>= 0) or a negative error code.
 * Thread-safe. */
WFA_API int64_t wfa_server_submit(wfa_server_t* s, const uint8_t* pattern, int32_t pattern_length,
                                  const uint8_t* text, int32_t text_length);
/* Moves up to `max` finished requests into `out` (their CIGAR ops densely
 * into `cigars`, at most cigar_cap bytes), waiting up to timeout_ms for the
 * first one.  Returns the count (0 on timeout) or a negative error code.
 * Thread-safe. */
WFA_API int32_t wfa_server_poll(wfa_server_t* s, wfa_served_t* out, int32_t max, uint8_t* cigars,
                                int64_t cigar_cap, int32_t timeout_ms);
/* Message of the last batch that failed (its requests carry the error code
 * as their status); "" if none.  Valid until the next failure. */
WFA_API const char* wfa_server_last_error(wfa_server_t* s);
/* Requests submitted and not yet polled. */
WFA_API int64_t wfa_server_pending(wfa_server_t* s);
/* Finishes the queued requests, stops the workers and frees the server. */
WFA_API int wfa_server_stop(wfa_server_t* s);

/* ---- resident stream: a persistent kernel fed request by request ----------
 * No counterpart in the reference.  One kernel stays on the GPU and aligns
 * single requests (end-to-end, high memory, n + m up to max_len_sum <= 2048,
 * ASCII bytes) as they are submitted: the host appends each request to a
 * ring in mapped pinned memory (capacity requests) and publishes it; one warp
 * of the kernel watches the ring's tail and every other lane group claims
 * the next request, aligns it with the batch kernels' per-pair aligner and
 * writes its result and CIGAR straight into mapped memory.  The kernel's
 * waits are bounded: it returns after about a second without requests (or
 * at wfa_stream_stop) and is launched again by the next submit or poll.  A
 * request that outgrows the kernel's scratch is aligned again through
 * wfa_batch_align.  Results are those of wfa_align_end2end with the same
 * metric, penalties and scope, whatever else is in flight.  The kernel holds
 * blocks_per_sm blocks on every SM (0: as many as fit) for as long as it
 * runs: work of other handles on the device shares what is left. */
typedef struct wfa_stream wfa_stream_t;
WFA_API wfa_stream_t* wfa_stream_start(wfa_metric_t metric, const wfa_penalties_t* penalties, int32_t device,
                                       int32_t score_only, int32_t max_len_sum, int32_t capacity,
                                       int32_t blocks_per_sm, int* err);
/* Queues one pair (copied into the ring); returns its id (ids count up from
 * 0), WFA_ERR_BUSY when capacity requests are outstanding, or an error. */
WFA_API int64_t wfa_stream_submit(wfa_stream_t* s, const uint8_t* pattern, int32_t pattern_length,
                                  const uint8_t* text, int32_t text_length);
/* Queues `count` pairs (offsets into seq, as in wfa_batch_t with ASCII
 * bytes) as separate requests with consecutive ids; returns the first id.
 * All or none: WFA_ERR_BUSY if they do not all fit. */
WFA_API int64_t wfa_stream_submit_many(wfa_stream_t* s, const uint8_t* seq, const int64_t* p_off,
                                       const int32_t* p_len, const int64_t* t_off, const int32_t* t_len,
                                       int64_t count);
/* Moves up to `max` finished requests into `out` (CIGAR ops densely into
 * `cigars`, at most cigar_cap bytes; mode 0), waiting up to timeout_ms for
 * the first; latency_ns runs from submit to the poll that found the result.
 * Returns the count (0 on timeout) or an error code. */
WFA_API int32_t wfa_stream_poll(wfa_stream_t* s, wfa_served_t* out, int32_t max, uint8_t* cigars,
                                int64_t cigar_cap, int32_t timeout_ms);
/* Requests submitted and not yet polled. */
WFA_API int64_t wfa_stream_pending(wfa_stream_t* s);
/* Up to n of: kernel launches, launches that ended idle, lane groups that
 * gave up polling, requests re-aligned through wfa_batch_align, blocks, lanes
 * per request. */
WFA_API int wfa_stream_stats(wfa_stream_t* s, int64_t* out, int32_t n);
/* Aligns what was submitted, ends the kernel and frees the stream (results
 * not yet polled are dropped). */
WFA_API int wfa_stream_stop(wfa_stream_t* s);

/* Device-checks build only (libwfa_b200_checked.so, WFA_DEVICE_CHECKS): the
 * number of failed index checks of the aligner's invariants in this
 * handle's kernels so far (each failure skips the access or re-runs the
 * pair); -1 from the product build, which compiles the checks out.  No
 * counterpart in the reference (its debug builds assert). */
WFA_API int64_t wfa_device_check_failures(wfa_aligner_t* h);

/* Number of the library's own kernel launches issued so far by this handle. */
WFA_API int64_t wfa_kernel_launches(const wfa_aligner_t* h);

/* Pairs the handle's last batch call re-ran with larger scratch (a pair
 * re-run twice counts twice); 0 when every pair finished in the first
 * launch.  No counterpart in the reference (it has no device scratch). */
WFA_API int64_t wfa_last_rerun_pairs(const wfa_aligner_t* h);

/* Lanes per pair of the unidirectional kernel for end-to-end alignments
 * without a heuristic: 4, 8, 16 or 32 (a lane group of that width aligns one
 * pair; 32 / lanes pairs share a warp), or 0 (the default) for the
 * autotuned choice.  The first device batch of each kind (device, metric,
 * encoding, score-only or CIGAR, length bucket n + m <= 384 / 1024 / 2048)
 * in a process times the candidates on a sample of its pairs and keeps the
 * fastest; ends-free, heuristic and med/low alignments and pairs above
 * n + m = 2048 always take whole warps.  Results never depend on it.  No
 * counterpart in the reference (it aligns one pair per call on the CPU). */
WFA_API int wfa_set_lanes_per_pair(wfa_aligner_t* h, int32_t lanes);
/* Lanes per pair of the BiWFA kernel: 32 (a warp aligns one pair), 128, 256
 * or 512 (a team of 4, 8 or 16 warps of one block aligns one pair; their
 * collectives meet at a named barrier), or 0 (the default) to choose by the
 * launch's longest pair (n + m above 3000: 256; above 1000: 128; else 32).  Teams run the kernels without a heuristic; with a
 * heuristic the BiWFA kernel always takes a warp per pair.  Results never
 * depend on it.  No counterpart in the reference. */
WFA_API int wfa_set_biwfa_lanes(wfa_aligner_t* h, int32_t lanes);
/* Lanes per pair the handle's last batch ran with (first round). */
WFA_API int32_t wfa_last_lanes_per_pair(const wfa_aligner_t* h);
/* Device memory (bytes) one pair in flight used in the handle's last
 * unidirectional launch: its lane group's scratch slice (ring cells beyond
 * shared memory, the high-memory M history or the med/low backtrace
 * buffer).  No counterpart in the reference. */
WFA_API int64_t wfa_last_slice_bytes(const wfa_aligner_t* h);
/* The autotuner's choices so far, one line per kind with the candidates'
 * sample times, into out (NUL-terminated, at most cap bytes); returns the
 * full length. */
WFA_API int32_t wfa_autotune_report(char* out, int32_t cap);

/* Device time (ms, CUDA events on the launching stream) of the alignment
 * kernel launches of the handle's last call, retries included. */
WFA_API double wfa_last_kernel_ms(const wfa_aligner_t* h);

/* ---- helpers -------------------------------------------------------------- */

/* Cigar::to_string_rle(true), src/cigar.rs:522-546.  Writes at most cap-1
 * chars and a NUL; returns the full string length. */
WFA_API int32_t wfa_cigar_rle(const uint8_t* ops, int32_t length, char* out, int32_t cap);

/* Library version string. */
WFA_API const char* wfa_version(void);

#ifdef __cplusplus
}
#endif
#endif /* WFA_B200_H */
