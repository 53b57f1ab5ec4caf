"""Python mirror of the wfa2lib-rs aligner API over the C ABI (include/wfa_b200.h).

`WavefrontAligner` has the methods of the reference's WavefrontAligner
(src/aligner.rs:407-3555) with the same names, argument meaning and results;
where the reference panics (invalid penalties) this raises ValueError.  Every
alignment runs in the CUDA library (lib/libwfa_b200.so); if it is missing or no
GPU is present the calls raise -- there is no CPU path.

Batches: `align_batch` (host arrays; copies in and out) and
`align_batch_device` (device pointers, e.g. torch CUDA tensors; no copies).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# WFA_B200_CHECKED=1 loads the device-checks build (tests only; make checked).
LIB_PATH = os.path.join(_HERE, "lib", "libwfa_b200_checked.so" if os.environ.get("WFA_B200_CHECKED") == "1"
                        else "libwfa_b200.so")

# Enum values of include/wfa_b200.h (the reference's enum order).
INDEL, EDIT, GAP_LINEAR, GAP_AFFINE, GAP_AFFINE_2P = range(5)
STATUS_NAMES = ["Ok", "EndReached", "EndUnreachable", "MaxStepsReached", "Oom", "Completed",
                "Partial"]
OK, END_REACHED, END_UNREACHABLE, MAX_STEPS_REACHED, OOM, COMPLETED, PARTIAL = range(7)
SCOPE_SCORE, SCOPE_ALIGNMENT = 0, 1
MEMORY = {"high": 0, "med": 1, "low": 2}
HEURISTICS = {"none": 0, "wfa-adaptive": 1, "xdrop": 2, "zdrop": 3, "banded-static": 4,
              "banded-adaptive": 5}
SEQ_ASCII, SEQ_PACKED2 = 0, 1
SPAN_END2END, SPAN_ENDSFREE = 0, 1
ERRORS = {-1: "invalid penalties", -2: "invalid argument", -3: "unsupported configuration",
          -4: "CUDA error", -5: "no CUDA device", -6: "out of device memory", -7: "stream ring full"}

RESULT_DTYPE = np.dtype([(f, np.int32) for f in (
    "score", "status", "cigar_begin", "cigar_length", "cigar_score", "end_v", "end_h",
    "end_score", "end_k", "end_offset")])


class Penalties(ctypes.Structure):
    _fields_ = [("match", ctypes.c_int32), ("mismatch", ctypes.c_int32),
                ("gap_opening1", ctypes.c_int32), ("gap_extension1", ctypes.c_int32),
                ("gap_opening2", ctypes.c_int32), ("gap_extension2", ctypes.c_int32)]


class Batch(ctypes.Structure):
    _fields_ = [("format", ctypes.c_int32), ("span", ctypes.c_int32), ("num_pairs", ctypes.c_int64),
                ("seq", ctypes.c_void_p), ("seq_bytes", ctypes.c_int64),
                ("p_off", ctypes.c_void_p), ("p_len", ctypes.c_void_p),
                ("t_off", ctypes.c_void_p), ("t_len", ctypes.c_void_p),
                ("cigar_off", ctypes.c_void_p), ("cigar_bytes", ctypes.c_int64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("metric", ctypes.c_int32), ("penalties", Penalties), ("device", ctypes.c_int32),
                ("score_only", ctypes.c_int32), ("workers", ctypes.c_int32),
                ("max_batch_pairs", ctypes.c_int32), ("max_batch_bytes", ctypes.c_int64),
                ("biwfa_above_bytes", ctypes.c_int64), ("short_workers", ctypes.c_int32),
                ("biwfa_workers", ctypes.c_int32), ("short_max_len", ctypes.c_int32),
                ("resident", ctypes.c_int32)]


class Served(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("score", ctypes.c_int32), ("status", ctypes.c_int32),
                ("cigar_length", ctypes.c_int32), ("cigar_score", ctypes.c_int32),
                ("end_v", ctypes.c_int32), ("end_h", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("cigar_offset", ctypes.c_int64),
                ("latency_ns", ctypes.c_int64)]


_lib = None


def lib():
    """The CUDA library; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    P32 = ctypes.POINTER(i32)
    sig = {
        "wfa_penalties_check": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Penalties)]),
        "wfa_aligner_create": (vp, [ctypes.c_int, ctypes.POINTER(Penalties), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int)]),
        "wfa_aligner_destroy": (None, [vp]),
        "wfa_set_memory_mode": (ctypes.c_int, [vp, ctypes.c_int]),
        "wfa_set_max_memory_compact": (ctypes.c_int, [vp, ctypes.c_uint64]),
        "wfa_set_max_alignment_steps": (ctypes.c_int, [vp, i32]),
        "wfa_set_alignment_scope": (ctypes.c_int, [vp, ctypes.c_int]),
        "wfa_set_alignment_free_ends": (ctypes.c_int, [vp, i32, i32, i32, i32]),
        "wfa_set_alignment_extension": (ctypes.c_int, [vp]),
        "wfa_set_alignment_end_to_end": (ctypes.c_int, [vp]),
        "wfa_set_compat": (ctypes.c_int, [vp, ctypes.c_int]),
        "wfa_set_heuristic": (ctypes.c_int, [vp, ctypes.c_int, i32, i32, i32]),
        "wfa_status": (ctypes.c_int, [vp]),
        "wfa_cigar": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_void_p), P32, P32, P32, P32]),
        "wfa_alignment_end_pos": (ctypes.c_int, [vp, P32, P32, P32]),
        "wfa_last_error": (ctypes.c_int, [vp]),
        "wfa_last_error_string": (ctypes.c_char_p, [vp]),
        "wfa_batch_align": (ctypes.c_int, [vp, ctypes.POINTER(Batch), vp, vp]),
        "wfa_batch_align_device": (ctypes.c_int, [vp, ctypes.POINTER(Batch), vp, vp, vp]),
        "wfa_batch_submit": (i64, [vp, ctypes.POINTER(Batch), vp, vp]),
        "wfa_batch_poll": (ctypes.c_int, [vp, i64, ctypes.POINTER(ctypes.c_int)]),
        "wfa_batch_wait": (ctypes.c_int, [vp, i64]),
        "wfa_batch_align_device_noalloc": (ctypes.c_int, [vp, ctypes.POINTER(Batch), vp, vp, vp]),
        "wfa_server_start": (vp, [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_int)]),
        "wfa_server_submit": (i64, [vp, ctypes.c_char_p, i32, ctypes.c_char_p, i32]),
        "wfa_server_poll": (i32, [vp, ctypes.POINTER(Served), i32, vp, i64, i32]),
        "wfa_server_last_error": (ctypes.c_char_p, [vp]),
        "wfa_server_pending": (i64, [vp]),
        "wfa_server_stop": (ctypes.c_int, [vp]),
        "wfa_stream_start": (vp, [ctypes.c_int, ctypes.POINTER(Penalties), i32, i32, i32, i32, i32,
                                  ctypes.POINTER(ctypes.c_int)]),
        "wfa_stream_submit": (i64, [vp, ctypes.c_char_p, i32, ctypes.c_char_p, i32]),
        "wfa_stream_submit_many": (i64, [vp, vp, vp, vp, vp, vp, i64]),
        "wfa_stream_poll": (i32, [vp, ctypes.POINTER(Served), i32, vp, i64, i32]),
        "wfa_stream_pending": (i64, [vp]),
        "wfa_stream_stats": (ctypes.c_int, [vp, ctypes.POINTER(i64), i32]),
        "wfa_stream_stop": (ctypes.c_int, [vp]),
        "wfa_kernel_launches": (i64, [vp]),
        "wfa_device_check_failures": (i64, [vp]),
        "wfa_last_rerun_pairs": (i64, [vp]),
        "wfa_set_lanes_per_pair": (ctypes.c_int, [vp, i32]),
        "wfa_last_lanes_per_pair": (i32, [vp]),
        "wfa_set_biwfa_lanes": (ctypes.c_int, [vp, i32]),
        "wfa_last_slice_bytes": (i64, [vp]),
        "wfa_autotune_report": (i32, [ctypes.c_char_p, i32]),
        "wfa_last_kernel_ms": (ctypes.c_double, [vp]),
        "wfa_cigar_rle": (i32, [vp, i32, ctypes.c_char_p, i32]),
        "wfa_version": (ctypes.c_char_p, []),
    }
    for name in ("wfa_align_end2end", "wfa_align_endsfree", "wfa_align_biwfa",
                 "wfa_align_biwfa_score", "wfa_align_packed2bits"):
        sig[name] = (i32, [vp, ctypes.c_char_p, i32, ctypes.c_char_p, i32])
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _pen(metric, penalties):
    p = list(penalties or []) + [0] * 6
    if metric == GAP_LINEAR:  # (match, mismatch, indel)
        return Penalties(p[0], p[1], p[2], 0, 0, 0)
    return Penalties(*p[:6])


class Cigar:
    """The reference's Cigar (src/cigar.rs:16): operations plus score/end."""

    def __init__(self, ops, score, end_v, end_h):
        self.operations = ops
        self.score, self.end_v, self.end_h = score, end_v, end_h

    def to_string_rle(self, print_matches=True):
        out, i, ops = [], 0, self.operations.decode()
        while i < len(ops):
            j = i
            while j < len(ops) and ops[j] == ops[i]:
                j += 1
            if print_matches or ops[i] != "M":
                out.append(f"{j - i}{ops[i]}")
            i = j
        return "".join(out)

    def is_null(self):
        return len(self.operations) == 0


class WavefrontAligner:
    """WavefrontAligner<N> (src/aligner.rs:146) backed by the B200 library."""

    def __init__(self, metric, penalties=None, device=0):
        L = lib()
        err = ctypes.c_int(0)
        self.metric = metric
        self.penalties = list(penalties or [])
        self._h = L.wfa_aligner_create(metric, ctypes.byref(_pen(metric, penalties)), device,
                                       ctypes.byref(err))
        if not self._h:
            if err.value == -1:
                raise ValueError(f"invalid penalties {penalties} for metric {metric}")
            raise RuntimeError(f"wfa_aligner_create failed: {ERRORS.get(err.value, err.value)}")
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            self._L.wfa_aligner_destroy(self._h)
            self._h = None

    __del__ = close

    def _check(self, r):
        if r < 0:
            msg = self._L.wfa_last_error_string(self._h).decode()
            if r == -3:
                raise NotImplementedError(msg)
            raise RuntimeError(f"{ERRORS.get(r, r)}: {msg}")
        return r

    # --- builder setters (src/aligner.rs:462-613) ---
    def set_memory_mode(self, mode):
        self._check(self._L.wfa_set_memory_mode(self._h, MEMORY.get(mode, mode)))

    def set_max_memory_compact(self, nbytes):
        self._check(self._L.wfa_set_max_memory_compact(self._h, nbytes))

    def set_max_alignment_steps(self, steps):
        self._check(self._L.wfa_set_max_alignment_steps(self._h, steps))

    def set_alignment_scope(self, compute_alignment):
        s = SCOPE_ALIGNMENT if compute_alignment in (True, SCOPE_ALIGNMENT) else SCOPE_SCORE
        self._check(self._L.wfa_set_alignment_scope(self._h, s))

    def set_alignment_free_ends(self, pattern_begin_free, pattern_end_free, text_begin_free,
                                text_end_free):
        self._check(self._L.wfa_set_alignment_free_ends(
            self._h, pattern_begin_free, pattern_end_free, text_begin_free, text_end_free))

    def set_alignment_extension(self):
        self._check(self._L.wfa_set_alignment_extension(self._h))

    def set_alignment_end_to_end(self):
        self._check(self._L.wfa_set_alignment_end_to_end(self._h))

    def set_compat(self, corrected):
        self._check(self._L.wfa_set_compat(self._h, 1 if corrected else 0))

    def set_heuristic(self, kind, *params):
        k = HEURISTICS[kind] if isinstance(kind, str) else (kind or 0)
        p = list(params) + [0, 0, 0]
        self._check(self._L.wfa_set_heuristic(self._h, k, p[0], p[1], p[2]))

    # --- plain per-call aligners ---
    def align_end2end(self, pattern, text):
        return self._check(self._L.wfa_align_end2end(self._h, pattern, len(pattern), text, len(text)))

    def align_endsfree(self, pattern, text):
        return self._check(self._L.wfa_align_endsfree(self._h, pattern, len(pattern), text, len(text)))

    def align_biwfa(self, pattern, text):
        return self._check(self._L.wfa_align_biwfa(self._h, pattern, len(pattern), text, len(text)))

    def align_biwfa_score(self, pattern, text):
        return self._check(self._L.wfa_align_biwfa_score(self._h, pattern, len(pattern), text,
                                                         len(text)))

    def align_packed2bits(self, pattern, pattern_length, text, text_length):
        return self._check(self._L.wfa_align_packed2bits(self._h, pattern, pattern_length, text,
                                                         text_length))

    def align_lambda(self, match_funct, pattern_length, text_length):
        raise NotImplementedError("lambda sequences need a host callback per base comparison")

    def status(self):
        return self._L.wfa_status(self._h)

    def cigar(self):
        ops = ctypes.c_void_p()
        n, s, v, h = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._L.wfa_cigar(self._h, ctypes.byref(ops), ctypes.byref(n), ctypes.byref(s),
                          ctypes.byref(v), ctypes.byref(h))
        data = ctypes.string_at(ops.value, n.value) if n.value > 0 else b""
        return Cigar(data, s.value, v.value, h.value)

    @property
    def alignment_end_pos(self):
        s, k, o = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._L.wfa_alignment_end_pos(self._h, ctypes.byref(s), ctypes.byref(k), ctypes.byref(o))
        return s.value, k.value, o.value

    def kernel_launches(self):
        return self._L.wfa_kernel_launches(self._h)

    def last_kernel_ms(self):
        return self._L.wfa_last_kernel_ms(self._h)

    def last_rerun_pairs(self):
        """Pairs the last batch call re-ran with larger scratch."""
        return self._L.wfa_last_rerun_pairs(self._h)

    def set_lanes_per_pair(self, lanes):
        """4, 8, 16 or 32 lanes per pair for end-to-end alignments without a
        heuristic, or 0 for the autotuned choice (the default)."""
        return self._check(self._L.wfa_set_lanes_per_pair(self._h, lanes))

    def set_biwfa_lanes(self, lanes):
        """32 lanes (a warp) or 128, 256, 512 (a team of warps) per pair for
        BiWFA batches without a heuristic; 0 chooses by the longest pair."""
        return self._check(self._L.wfa_set_biwfa_lanes(self._h, lanes))

    def device_check_failures(self):
        """Failed index checks in this handle's kernels (device-checks build),
        -1 with the product build."""
        return self._L.wfa_device_check_failures(self._h)

    def last_lanes_per_pair(self):
        return self._L.wfa_last_lanes_per_pair(self._h)

    def last_slice_bytes(self):
        """Device bytes one pair in flight used in the last launch."""
        return self._L.wfa_last_slice_bytes(self._h)

    # --- batches ---
    def align_batch(self, seq, p_off, p_len, t_off, t_len, packed=False, span=SPAN_END2END,
                    out_results=None, out_cigars=None):
        """Host arrays in; returns (results[RESULT_DTYPE], dense CIGAR bytes).

        Pair i's CIGAR is cigars[r['cigar_begin'] : r['cigar_begin'] + r['cigar_length']].
        out_results / out_cigars may be preallocated (e.g. pinned) buffers; the
        CIGAR buffer needs sum(2*(p_len+t_len)+1) bytes at most."""
        n = len(p_len)
        seq = np.ascontiguousarray(seq).view(np.uint8)
        arrs = [a if (isinstance(a, np.ndarray) and a.dtype == d and a.flags.c_contiguous)
                else np.ascontiguousarray(a, dtype=d) for a, d in
                ((p_off, np.int64), (p_len, np.int32), (t_off, np.int64), (t_len, np.int32))]
        res = out_results if out_results is not None else np.zeros(n, RESULT_DTYPE)
        if out_cigars is not None:
            cig = out_cigars
        else:
            caps = 2 * (arrs[1].astype(np.int64) + arrs[3]) + 1
            cig = np.zeros(int(caps.sum()) + 16, np.uint8)
        b = Batch(SEQ_PACKED2 if packed else SEQ_ASCII, span, n, seq.ctypes.data, seq.nbytes,
                  arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
                  arrs[3].ctypes.data, None, 0)
        self._check(self._L.wfa_batch_align(self._h, ctypes.byref(b), res.ctypes.data,
                                            cig.ctypes.data))
        return res, cig

    def submit_batch(self, seq, p_off, p_len, t_off, t_len, packed=False, span=SPAN_END2END):
        """align_batch without waiting: returns a ticket; wait_batch(ticket)
        returns (results, dense CIGAR bytes) as align_batch does."""
        n = len(p_len)
        seq = np.ascontiguousarray(seq).view(np.uint8)
        arrs = [np.ascontiguousarray(x, dtype=d) for x, d in
                ((p_off, np.int64), (p_len, np.int32), (t_off, np.int64), (t_len, np.int32))]
        res = np.zeros(n, RESULT_DTYPE)
        caps = 2 * (arrs[1].astype(np.int64) + arrs[3]) + 1
        cig = np.zeros(int(caps.sum()) + 16, np.uint8)
        b = Batch(SEQ_PACKED2 if packed else SEQ_ASCII, span, n, seq.ctypes.data, seq.nbytes,
                  arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
                  arrs[3].ctypes.data, None, 0)
        t = self._L.wfa_batch_submit(self._h, ctypes.byref(b), res.ctypes.data, cig.ctypes.data)
        self._check(t)
        if not hasattr(self, "_pending"):
            self._pending = {}
        self._pending[t] = (seq, arrs, res, cig)  # alive until the batch is done
        return t

    def poll_batch(self, ticket):
        """True once the ticket's batch is done (then wait_batch returns at once)."""
        st = ctypes.c_int(0)
        r = self._L.wfa_batch_poll(self._h, ticket, ctypes.byref(st))
        self._check(r)
        if r == 1:
            self._check(st.value)
            self._pending[ticket] = self._pending[ticket][2:] + ("done",)
        return r == 1

    def wait_batch(self, ticket):
        p = self._pending.pop(ticket)
        if len(p) == 3:  # already reported done by poll_batch
            return p[0], p[1]
        self._check(self._L.wfa_batch_wait(self._h, ticket))
        return p[2], p[3]

    def align_batch_device(self, seq_ptr, seq_bytes, p_off, p_len, t_off, t_len, num_pairs,
                           results_ptr, cigars_ptr=None, cigar_off=None, cigar_bytes=0,
                           packed=False, span=SPAN_END2END, stream=0):
        """All arguments are device pointers (ints); enqueued on `stream`."""
        b = Batch(SEQ_PACKED2 if packed else SEQ_ASCII, span, num_pairs, seq_ptr, seq_bytes,
                  p_off, p_len, t_off, t_len, cigar_off, cigar_bytes)
        return self._check(self._L.wfa_batch_align_device(self._h, ctypes.byref(b), results_ptr,
                                                          cigars_ptr, stream))

    def align_batch_device_noalloc(self, seq_ptr, seq_bytes, p_off, p_len, t_off, t_len,
                                   num_pairs, results_ptr, cigars_ptr=None, cigar_off=None,
                                   cigar_bytes=0, packed=False, span=SPAN_END2END, stream=0):
        """align_batch_device without any device allocation: for callers that
        must not allocate device memory (their own allocator holds it, or a
        cudaFree would stall their other streams).  Scratch is one fixed
        64 MiB device array shared by all calls on a device, so calls that
        overlap on the GPU race; the longest pair may have n + m <= 4096."""
        b = Batch(SEQ_PACKED2 if packed else SEQ_ASCII, span, num_pairs, seq_ptr, seq_bytes,
                  p_off, p_len, t_off, t_len, cigar_off, cigar_bytes)
        return self._check(self._L.wfa_batch_align_device_noalloc(
            self._h, ctypes.byref(b), results_ptr, cigars_ptr, stream))


class Server:
    """Continuous-batching request loop over the GPU (wfa_server_* of the C
    ABI): submit single pairs from any thread, poll finished ones.  Requests
    go to a short, a long high-memory or a BiWFA lane; a request runs BiWFA
    when its predicted high-memory footprint ((n + m)^2 / 4 bytes) exceeds
    `biwfa_above_bytes`.  Either way its result is that of the plain aligner
    call in that mode, alone or in any mix."""

    def __init__(self, metric, penalties=None, device=0, score_only=False, workers=2,
                 max_batch_pairs=65536, max_batch_bytes=4 << 30, biwfa_above_bytes=256 << 20,
                 short_workers=2, biwfa_workers=2, short_max_len=1024, resident=False):
        self._L = lib()
        cfg = ServerConfig(metric, _pen(metric, penalties), device, int(score_only), workers,
                           max_batch_pairs, max_batch_bytes, biwfa_above_bytes, short_workers,
                           biwfa_workers, short_max_len, int(resident))
        err = ctypes.c_int(0)
        self._s = self._L.wfa_server_start(ctypes.byref(cfg), ctypes.byref(err))
        if not self._s:
            raise RuntimeError(f"wfa_server_start: {ERRORS.get(err.value, err.value)}")
        self._recs = (Served * 4096)()
        self._cig = ctypes.create_string_buffer(64 << 20)

    def submit(self, pattern, text):
        r = self._L.wfa_server_submit(self._s, pattern, len(pattern), text, len(text))
        if r < 0:
            raise RuntimeError(f"wfa_server_submit: {ERRORS.get(r, r)}")
        return r

    def poll(self, timeout_ms=100, max_records=4096):
        """Finished requests: list of dicts (id, score, status, cigar bytes,
        cigar_score, end_v, end_h, mode, latency_ns)."""
        c = self._L.wfa_server_poll(self._s, self._recs, min(max_records, 4096), self._cig,
                                    len(self._cig), timeout_ms)
        if c < 0:
            raise RuntimeError(f"wfa_server_poll: {ERRORS.get(c, c)}")
        out = []
        raw = self._cig.raw
        for i in range(c):
            r = self._recs[i]
            cig = raw[r.cigar_offset:r.cigar_offset + r.cigar_length] if r.cigar_offset >= 0 else b""
            out.append({"id": r.id, "score": r.score, "status": r.status, "cigar": cig,
                        "cigar_score": r.cigar_score, "end_v": r.end_v, "end_h": r.end_h,
                        "mode": r.mode, "latency_ns": r.latency_ns})
        return out

    def pending(self):
        return self._L.wfa_server_pending(self._s)

    def last_error(self):
        return self._L.wfa_server_last_error(self._s).decode()

    def stop(self):
        if self._s:
            self._L.wfa_server_stop(self._s)
            self._s = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


STREAM_DTYPE = np.dtype([("id", np.int64), ("score", np.int32), ("status", np.int32),
                         ("cigar_length", np.int32), ("cigar_score", np.int32), ("end_v", np.int32),
                         ("end_h", np.int32), ("mode", np.int32), ("pad", np.int32),
                         ("cigar_offset", np.int64), ("latency_ns", np.int64)])
assert STREAM_DTYPE.itemsize == ctypes.sizeof(Served)


class Stream:
    """A resident serving kernel fed request by request (wfa_stream_* of the
    C ABI): end-to-end alignments of pairs with n + m <= max_len_sum, each
    submitted on its own (or many at once, still separate requests) while
    the kernel runs; results are those of WavefrontAligner.align_end2end."""

    def __init__(self, metric, penalties=None, device=0, score_only=False, max_len_sum=512,
                 capacity=1 << 16, blocks_per_sm=0):
        self._L = lib()
        err = ctypes.c_int(0)
        pen = _pen(metric, penalties)
        self._s = self._L.wfa_stream_start(metric, ctypes.byref(pen), device, int(score_only),
                                           max_len_sum, capacity, blocks_per_sm, ctypes.byref(err))
        if not self._s:
            raise RuntimeError(f"wfa_stream_start: {ERRORS.get(err.value, err.value)}")
        self._max = 1 << 16
        self._recs = np.zeros(self._max, STREAM_DTYPE)
        self._cig = np.zeros(self._max * (2 * max_len_sum + 1), np.uint8)

    def submit(self, pattern, text):
        """One request; its id, or -7 (WFA_ERR_BUSY) when the ring is full."""
        r = self._L.wfa_stream_submit(self._s, pattern, len(pattern), text, len(text))
        if r < 0 and r != -7:
            raise RuntimeError(f"wfa_stream_submit: {ERRORS.get(r, r)}")
        return r

    def submit_many(self, seq, p_off, p_len, t_off, t_len):
        """Requests for pairs at byte offsets of seq (uint8); the first id
        (ids are consecutive), or -7 (WFA_ERR_BUSY) if they do not all fit."""
        seq = np.ascontiguousarray(seq, np.uint8)
        arrs = [np.ascontiguousarray(a, t) for a, t in ((p_off, np.int64), (p_len, np.int32),
                                                          (t_off, np.int64), (t_len, np.int32))]
        r = self._L.wfa_stream_submit_many(self._s, seq.ctypes.data, *[a.ctypes.data for a in arrs],
                                           len(arrs[1]))
        if r < 0 and r != -7:
            raise RuntimeError(f"wfa_stream_submit_many: {ERRORS.get(r, r)}")
        return r

    def poll_arrays(self, timeout_ms=100, max_records=1 << 16):
        """Finished requests as a structured array (STREAM_DTYPE) and the
        CIGAR byte buffer its cigar_offset fields index (valid until the next
        poll)."""
        c = self._L.wfa_stream_poll(self._s, self._recs.ctypes.data_as(ctypes.POINTER(Served)),
                                    min(max_records, self._max), self._cig.ctypes.data,
                                    len(self._cig), timeout_ms)
        if c < 0:
            raise RuntimeError(f"wfa_stream_poll: {ERRORS.get(c, c)}")
        return self._recs[:c].copy(), self._cig

    def poll(self, timeout_ms=100, max_records=4096):
        """Finished requests: list of dicts (id, score, status, cigar bytes,
        cigar_score, end_v, end_h, latency_ns)."""
        recs, cig = self.poll_arrays(timeout_ms, max_records)
        out = []
        for r in recs:
            o, n = int(r["cigar_offset"]), int(r["cigar_length"])
            out.append({"id": int(r["id"]), "score": int(r["score"]), "status": int(r["status"]),
                        "cigar": cig[o:o + n].tobytes() if o >= 0 else b"",
                        "cigar_score": int(r["cigar_score"]), "end_v": int(r["end_v"]),
                        "end_h": int(r["end_h"]), "latency_ns": int(r["latency_ns"])})
        return out

    def pending(self):
        return self._L.wfa_stream_pending(self._s)

    def stats(self):
        """Kernel launches, launches that ended idle, lane groups that gave up
        polling, requests re-aligned through the batch path, blocks, lanes."""
        v = (ctypes.c_int64 * 6)()
        self._L.wfa_stream_stats(self._s, v, 6)
        keys = ("launches", "idle_exits", "gave_up", "fallbacks", "blocks", "lanes")
        return dict(zip(keys, list(v)))

    def stop(self):
        if self._s:
            rc = self._L.wfa_stream_stop(self._s)
            self._s = None
            if rc != 0:
                raise RuntimeError(f"wfa_stream_stop: {ERRORS.get(rc, rc)}")

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def cigar_rle(ops):
    """Cigar::to_string_rle(true) through the library helper."""
    L = lib()
    n = L.wfa_cigar_rle(ops, len(ops), None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    L.wfa_cigar_rle(ops, len(ops), buf, n + 1)
    return buf.value.decode()


def autotune_report():
    """The lane-width autotuner's choices in this process, one line per kind."""
    L = lib()
    n = L.wfa_autotune_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    L.wfa_autotune_report(buf, n + 1)
    return buf.value.decode()
