"""TEST-ONLY: ctypes driver of the one-lane host build of the device aligner."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESULT_DTYPE = np.dtype([(f, np.int32) for f in (
    "score", "status", "cigar_begin", "cigar_length", "cigar_score", "end_v", "end_h",
    "end_score", "end_k", "end_offset")])
_L = {}
LANES = int(os.environ.get("WFA_EMU_LANES", "1"))


def lib(lanes=None):
    lanes = LANES if lanes is None else lanes
    if lanes not in _L:
        name = {32: "libwfa_emu32.so", 8: "libwfa_emu8.so",
                128: "libwfa_emu128.so"}.get(lanes, "libwfa_emu.so")
        path = os.path.join(HERE, "emu", "_build", name)
        if os.system(f"make -s -C {os.path.join(HERE, 'emu')}") != 0 or not os.path.exists(path):
            raise RuntimeError("cannot build the emulation library")
        L = ctypes.CDLL(path)
        L.wfa_emu_batch.restype = ctypes.c_int64
        _L[lanes] = L
    return _L[lanes]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def run(metric, pen, pairs, compute_alignment=True, span=0, extension=0, free=None, heuristic=0,
        hparams=(0, 0, 0), max_steps=2**31 - 1, packed=False, wmax=4096, hist_scores=1 << 16,
        hist_words=1 << 22, lanes=None, piggyback=False, compat=0, bt_limit=256 << 20,
        bt_cap=1 << 20, bt_probe=6000):
    """pairs: list of (bytes, bytes).  Returns (results, list of cigar strings).
    piggyback: med/low memory with an alignment (the piggyback backtrace):
    True or "med", or "low"; compat: 0 C, 1 Corrected; bt_limit: bytes of
    backtrace blocks above which the buffer is compacted (max_memory_compact);
    bt_cap: blocks of the backtrace buffer; bt_probe: scores between
    compaction probes (the library's is the reference's 6000)."""
    n = len(pairs)
    if packed:
        words, p_off, t_off, p_len, t_len = [], [], [], [], []
        code = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3}
        pos = 0
        for p, t in pairs:
            for s, offs, lens in ((p, p_off, p_len), (t, t_off, t_len)):
                nw = (len(s) + 15) // 16
                w = np.zeros(nw * 16, np.uint32)
                w[:len(s)] = [code.get(c, 0) for c in s]
                packed_w = np.bitwise_or.reduce(w.reshape(-1, 16) << (2 * np.arange(16, dtype=np.uint32)), axis=1) if nw else np.zeros(0, np.uint32)
                words.append(packed_w.astype(np.uint32))
                offs.append(pos)
                lens.append(len(s))
                pos += nw
        seq = np.concatenate(words + [np.zeros(4, np.uint32)]).view(np.uint8)
    else:
        buf, p_off, t_off, p_len, t_len = bytearray(), [], [], [], []
        for p, t in pairs:
            p_off.append(len(buf)); buf += p; p_len.append(len(p))
            t_off.append(len(buf)); buf += t; t_len.append(len(t))
        buf += b"\0" * 16
        seq = np.frombuffer(bytes(buf), np.uint8).copy()
    p_off = np.array(p_off, np.int64); t_off = np.array(t_off, np.int64)
    p_len = np.array(p_len, np.int32); t_len = np.array(t_len, np.int32)
    caps = 2 * (p_len.astype(np.int64) + t_len) + 1
    c_off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    cig = np.zeros(int(caps.sum()) + 1, np.uint8)
    res = np.zeros(n, RESULT_DTYPE)
    pen6 = np.array(list(pen or []) + [0] * (6 - len(pen or [])), np.int32)
    free4 = np.array(list(free) if free else [0, 0, 0, 0], np.int32)
    hp3 = np.array(list(hparams) + [0] * (3 - len(hparams)), np.int32)
    L = lib(lanes)
    r = L.wfa_emu_batch(metric, _p(pen6), int(compute_alignment), span, extension, _p(free4),
                        heuristic, _p(hp3), ctypes.c_int32(max_steps), 1 if packed else 0,
                        _p(seq), ctypes.c_int64(seq.nbytes), _p(p_off), _p(p_len), _p(t_off),
                        _p(t_len), ctypes.c_int64(n), _p(c_off), _p(cig), _p(res),
                        ctypes.c_int32(wmax), ctypes.c_int32(hist_scores), ctypes.c_int64(hist_words),
                        2 if piggyback == "low" else int(bool(piggyback)), int(compat),
                        ctypes.c_int64(bt_limit), ctypes.c_int32(bt_cap), ctypes.c_int32(bt_probe))
    assert r >= 0
    cigars = []
    for i in range(n):
        b, l = res["cigar_begin"][i], res["cigar_length"][i]
        cigars.append(cig[c_off[i] + b: c_off[i] + b + l].tobytes().decode())
    return res, cigars


def run_biwfa(metric, pen, pairs, compute_alignment=True, heuristic=0, hparams=(0, 0, 0),
              max_steps=2**31 - 1, packed=False, wmax=4096, hist_scores=1 << 16, hist_words=1 << 22,
              lanes=None, idc=0):
    """BiWFA through the emulated device driver: (results, cigar strings).
    idc: the growth phase's I/D rings, 0 by length, 1 kept until the overlap
    scans (every search restarts), 2 off."""
    n = len(pairs)
    if packed:
        words, p_off, t_off, p_len, t_len = [], [], [], [], []
        code = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3}
        pos = 0
        for p, t in pairs:
            for s, offs, lens in ((p, p_off, p_len), (t, t_off, t_len)):
                nw = (len(s) + 15) // 16
                w = np.zeros(nw * 16, np.uint32)
                w[:len(s)] = [code.get(c, 0) for c in s]
                packed_w = np.bitwise_or.reduce(w.reshape(-1, 16) << (2 * np.arange(16, dtype=np.uint32)), axis=1) if nw else np.zeros(0, np.uint32)
                words.append(packed_w.astype(np.uint32))
                offs.append(pos)
                lens.append(len(s))
                pos += nw
        seq = np.concatenate(words + [np.zeros(4, np.uint32)]).view(np.uint8)
    else:
        buf, p_off, t_off, p_len, t_len = bytearray(), [], [], [], []
        for p, t in pairs:
            p_off.append(len(buf)); buf += p; p_len.append(len(p))
            t_off.append(len(buf)); buf += t; t_len.append(len(t))
        buf += b"\0" * 16
        seq = np.frombuffer(bytes(buf), np.uint8).copy()
    p_off = np.array(p_off, np.int64); t_off = np.array(t_off, np.int64)
    p_len = np.array(p_len, np.int32); t_len = np.array(t_len, np.int32)
    caps = 2 * (p_len.astype(np.int64) + t_len) + 1
    c_off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    cig = np.zeros(int(caps.sum()) + 1, np.uint8)
    res = np.zeros(n, RESULT_DTYPE)
    pen6 = np.array(list(pen or []) + [0] * (6 - len(pen or [])), np.int32)
    hp3 = np.array(list(hparams) + [0] * (3 - len(hparams)), np.int32)
    L = lib(lanes)
    L.wfa_emu_biwfa.restype = ctypes.c_int64
    r = L.wfa_emu_biwfa(metric, _p(pen6), int(compute_alignment), heuristic, _p(hp3),
                        ctypes.c_int32(max_steps), 1 if packed else 0, _p(seq), _p(p_off), _p(p_len),
                        _p(t_off), _p(t_len), ctypes.c_int64(n), _p(c_off), _p(cig), _p(res),
                        ctypes.c_int32(wmax), ctypes.c_int32(hist_scores), ctypes.c_int64(hist_words),
                        ctypes.c_int32(idc))
    assert r >= 0
    cigars = []
    for i in range(n):
        b, l = res["cigar_begin"][i], res["cigar_length"][i]
        cigars.append(cig[c_off[i] + b: c_off[i] + b + l].tobytes().decode())
    return res, cigars
