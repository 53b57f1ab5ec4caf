"""ctypes wrapper of the CPU oracle (oracle/wfa_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker / baseline, never by the product.
Build it with `make -C oracle` (done by __graft_entry__.build()).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
METRICS = {"indel-wfa": 0, "edit-wfa": 1, "gap-linear-wfa": 2, "gap-affine-wfa": 3,
           "gap-affine2p-wfa": 4}
# align_benchmark defaults, src/bin/align_benchmark.rs:148-220
DEFAULT_PEN = {0: [], 1: [], 2: [0, 4, 2], 3: [0, 4, 6, 2], 4: [0, 4, 6, 2, 24, 1]}
HEURISTICS = {None: 0, "none": 0, "wfa-adaptive": 1, "xdrop": 2, "zdrop": 3,
              "banded-static": 4, "banded-adaptive": 5}
STATUS = ["Ok", "EndReached", "EndUnreachable", "MaxStepsReached", "Oom", "Completed", "Partial"]

_lib = {}


def lib(fast=False):
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name in _lib:
        return _lib[name]
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        raise RuntimeError(f"oracle not built: {path} (run `make -C oracle`)")
    L = ctypes.CDLL(path)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    P32, P64 = ctypes.POINTER(i32), ctypes.POINTER(i64)
    L.wfo_create.restype = vp
    L.wfo_create.argtypes = [ctypes.c_int, P32]
    L.wfo_destroy.argtypes = [vp]
    L.wfo_set_alignment_scope.argtypes = [vp, ctypes.c_int]
    L.wfo_set_memory_mode.argtypes = [vp, ctypes.c_int]
    L.wfo_set_compat.argtypes = [vp, ctypes.c_int]
    L.wfo_set_piggyback_literal.argtypes = [vp, ctypes.c_int]
    L.wfo_set_heuristic.argtypes = [vp, ctypes.c_int, i32, i32, i32]
    L.wfo_set_max_alignment_steps.argtypes = [vp, i32]
    L.wfo_set_alignment_free_ends.argtypes = [vp, i32, i32, i32, i32]
    L.wfo_set_alignment_extension.argtypes = [vp]
    L.wfo_set_alignment_end_to_end.argtypes = [vp]
    for f in ("wfo_align_end2end", "wfo_align_endsfree", "wfo_align_biwfa", "wfo_align_biwfa_score"):
        getattr(L, f).argtypes = [vp, ctypes.c_char_p, i32, ctypes.c_char_p, i32]
        getattr(L, f).restype = i32
    L.wfo_align_packed2bits.argtypes = [vp, ctypes.c_char_p, i32, ctypes.c_char_p, i32]
    L.wfo_align_packed2bits.restype = i32
    L.wfo_status.argtypes = [vp]
    L.wfo_cigar.argtypes = [vp, ctypes.c_char_p, i32, P32, P32, P32]
    L.wfo_cigar.restype = i32
    L.wfo_end_pos.argtypes = [vp, P32, P32, P32]
    L.wfo_counters.argtypes = [vp, P64, P64, P64]
    L.wfo_cli_line.argtypes = [vp, ctypes.c_int, P32, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                               i32, ctypes.c_char_p, i32, ctypes.c_char_p, i32]
    L.wfo_cli_line.restype = i32
    L.wfo_batch.argtypes = [ctypes.c_int, P32, ctypes.c_int, ctypes.c_int, ctypes.c_int, P32, P32,
                            ctypes.c_char_p, P64, P32, P64, P32, i64, ctypes.c_int, P32, P32, P64,
                            P64]
    L.wfo_batch.restype = ctypes.c_double
    L.wfo_hash_ops.argtypes = [vp, P64, P32, i64, ctypes.c_int, P64]
    _lib[name] = L
    return L


def _arr(vals, n=6):
    vals = list(vals) + [0] * (n - len(vals))
    return (ctypes.c_int32 * n)(*vals)


class OracleAligner:
    """Mirror of the reference's WavefrontAligner builder (src/aligner.rs:146)."""

    def __init__(self, metric, penalties=None, fast=False):
        self.L = lib(fast)
        self.metric = metric
        pen = DEFAULT_PEN[metric] if penalties is None else list(penalties)
        self.h = self.L.wfo_create(metric, _arr(pen))
        if not self.h:
            raise ValueError(f"invalid penalties {pen} for metric {metric}")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.wfo_destroy(self.h)
            self.h = None

    def set_alignment_scope(self, compute_alignment):
        self.L.wfo_set_alignment_scope(self.h, 1 if compute_alignment else 0)

    def set_memory_mode(self, mode):
        self.L.wfo_set_memory_mode(self.h, {"high": 0, "med": 1, "low": 2}.get(mode, mode))

    def set_piggyback_literal(self, on):
        """Med/low: the reference's per-cell packed-CIGAR path (True, the
        default) or the picks re-made from the kept offsets (False)."""
        self.L.wfo_set_piggyback_literal(self.h, int(bool(on)))

    def set_compat(self, compat):
        """'c' (reproduce C's known bugs, the default) or 'corrected'."""
        self.L.wfo_set_compat(self.h, {"c": 0, "corrected": 1}.get(compat, compat))

    def set_heuristic(self, kind, *params):
        k = HEURISTICS[kind] if isinstance(kind, str) or kind is None else kind
        p = list(params) + [0] * (3 - len(params))
        self.L.wfo_set_heuristic(self.h, k, p[0], p[1], p[2])

    def set_max_alignment_steps(self, s):
        self.L.wfo_set_max_alignment_steps(self.h, s)

    def set_alignment_free_ends(self, p0, pf, t0, tf):
        self.L.wfo_set_alignment_free_ends(self.h, p0, pf, t0, tf)

    def set_alignment_extension(self):
        self.L.wfo_set_alignment_extension(self.h)

    def set_alignment_end_to_end(self):
        self.L.wfo_set_alignment_end_to_end(self.h)

    def align_end2end(self, p, t):
        return self.L.wfo_align_end2end(self.h, p, len(p), t, len(t))

    def align_endsfree(self, p, t):
        return self.L.wfo_align_endsfree(self.h, p, len(p), t, len(t))

    def align_biwfa(self, p, t):
        return self.L.wfo_align_biwfa(self.h, p, len(p), t, len(t))

    def align_biwfa_score(self, p, t):
        return self.L.wfo_align_biwfa_score(self.h, p, len(p), t, len(t))

    def align_packed2bits(self, p, n, t, m):
        return self.L.wfo_align_packed2bits(self.h, p, n, t, m)

    def status(self):
        return self.L.wfo_status(self.h)

    def cigar(self):
        """(ops bytes, score, end_v, end_h) of the last alignment."""
        s, v, hh = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        n = self.L.wfo_cigar(self.h, None, 0, ctypes.byref(s), ctypes.byref(v), ctypes.byref(hh))
        buf = ctypes.create_string_buffer(max(n, 1))
        self.L.wfo_cigar(self.h, buf, n, None, None, None)
        return buf.raw[:n], s.value, v.value, hh.value

    def end_pos(self):
        s, k, o = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self.L.wfo_end_pos(self.h, ctypes.byref(s), ctypes.byref(k), ctypes.byref(o))
        return s.value, k.value, o.value

    def counters(self):
        c, b, o = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.L.wfo_counters(self.h, ctypes.byref(c), ctypes.byref(b), ctypes.byref(o))
        return c.value, b.value, o.value

    def cli_line(self, p, t, span=0, free=None, biwfa=False, score_only=False):
        cap = 4 * (len(p) + len(t)) + 64
        buf = ctypes.create_string_buffer(cap)
        n = self.L.wfo_cli_line(self.h, span, _arr(free or [], 4), int(biwfa), int(score_only), p,
                                len(p), t, len(t), buf, cap)
        return None if n < 0 else buf.value.decode()


def nominal_prop(base, factor):
    """src/bin/align_benchmark.rs:257-263"""
    if 0.0 <= factor <= 1.0:
        return int(base * factor) & 0xFFFFFFFF
    return int(factor) & 0xFFFFFFFF


def run_cli_case(case, fast=False):
    """Run an align_benchmark-style case (as in tests/golden) through the oracle.

    Returns the output lines, or None where the driver exits with an error.
    """
    metric = METRICS[case["algo"]]
    pen = None
    if case.get("penalties"):
        pen = [int(x) for x in case["penalties"].split(",")]
    a = OracleAligner(metric, pen, fast=fast)
    score_only = bool(case.get("score_only"))
    if not score_only:
        a.set_alignment_scope(True)
    if case.get("no_c_compat"):
        a.set_compat("corrected")
    mem = case.get("memory", "high")
    biwfa = mem == "ultralow"
    a.set_memory_mode("high" if biwfa else mem)
    span_s = case.get("span", "global")
    if span_s == "global":
        span, fracs = 0, None
    elif span_s in ("extension", "extend"):
        span, fracs = 1, None
        a.set_alignment_extension()
    else:
        span, fracs = 2, [float(x) for x in span_s.split(",")[1:]]
    h = case.get("heuristic")
    if h and h != "none":
        params = [int(x) for x in case["hparams"].split(",")]
        if h in ("xdrop", "zdrop") and (biwfa or metric in (0, 1)):
            return None
        a.set_heuristic(h, *params)
    lines = []
    for p, t in case["pairs"]:
        pb, tb = p.encode(), t.encode()
        free = None
        if span == 2:
            free = [nominal_prop(len(pb), fracs[0]), nominal_prop(len(pb), fracs[1]),
                    nominal_prop(len(tb), fracs[2]), nominal_prop(len(tb), fracs[3])]
        line = a.cli_line(pb, tb, span=span, free=free, biwfa=biwfa, score_only=score_only)
        if line is None:
            return lines if lines else None
        lines.append(line)
    return lines


def batch(metric, penalties, seqbuf, p_off, p_len, t_off, t_len, compute_alignment=True, mode=0,
          heuristic=0, hparams=(0, 0, 0), free=None, threads=1, want_results=True, work=None):
    """Multi-threaded batch over the fast build; returns (seconds, scores, status, cigar_hash).
    work: an int64 array of 3 that receives the batch's summed work counters
    (cells computed, bases compared, CIGAR ops)."""
    import numpy as np
    L = lib(fast=True)
    n = len(p_len)
    P32 = ctypes.POINTER(ctypes.c_int32)
    P64 = ctypes.POINTER(ctypes.c_int64)
    p_off = np.ascontiguousarray(p_off, dtype=np.int64)
    t_off = np.ascontiguousarray(t_off, dtype=np.int64)
    p_len = np.ascontiguousarray(p_len, dtype=np.int32)
    t_len = np.ascontiguousarray(t_len, dtype=np.int32)
    scores = np.zeros(n, np.int32) if want_results else None
    status = np.zeros(n, np.int32) if want_results else None
    hashes = np.zeros(n, np.int64) if want_results else None
    pen = DEFAULT_PEN[metric] if penalties is None else penalties
    secs = L.wfo_batch(metric, _arr(pen), int(compute_alignment), mode, heuristic,
                       _arr(hparams, 3), _arr(free, 4) if free is not None else None,
                       seqbuf, p_off.ctypes.data_as(P64), p_len.ctypes.data_as(P32),
                       t_off.ctypes.data_as(P64), t_len.ctypes.data_as(P32), n, threads,
                       scores.ctypes.data_as(P32) if want_results else None,
                       status.ctypes.data_as(P32) if want_results else None,
                       hashes.ctypes.data_as(P64) if want_results else None,
                       work.ctypes.data_as(P64) if work is not None else None)
    return secs, scores, status, hashes


def hash_ops(ops, begin, length, threads=1):
    """FNV-1a hashes of ops[begin[i]:begin[i]+length[i]] (uint8 array), the
    hash `batch` reports per CIGAR."""
    import numpy as np
    ops = np.ascontiguousarray(ops, dtype=np.uint8)
    begin = np.ascontiguousarray(begin, dtype=np.int64)
    length = np.ascontiguousarray(length, dtype=np.int32)
    out = np.zeros(len(begin), np.int64)
    L = lib(fast=True)
    L.wfo_hash_ops(ctypes.c_void_p(ops.ctypes.data), begin.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                   length.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(begin), threads,
                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out
