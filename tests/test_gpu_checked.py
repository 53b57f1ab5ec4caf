"""The device-checks build (libwfa_b200_checked.so: the library compiled with
WFA_DEVICE_CHECKS, which counts failed index checks of the aligner's
invariants instead of compiling them out) on the GPU: across the batch
forms, metrics and lane widths no check fails, and every result equals the
oracle's.  The build is loaded in a child process (one library per
process)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r'''
import os, random, sys
import numpy as np
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from _pkg import load
import oracle as O
from test_gpu_parity import pack
from test_emu_biwfa import long_pairs
pkg = load()
from wfa_b200 import synth
total = 0

def check(a, res, cig, metric, pen, pairs, mode, span, hk=0, hp=(0, 0, 0)):
    global total
    n = a.device_check_failures()
    assert n == 0, ("failed checks", n, metric, mode, span)
    for i, (p, t) in enumerate(pairs):
        o = O.OracleAligner(metric, pen)
        o.set_alignment_scope(True)
        o.set_memory_mode(mode)
        if hk:
            o.set_heuristic(hk, *hp)
        if span == 1:
            o.set_alignment_free_ends(len(p) // 5, len(p) // 5, len(t) // 5, len(t) // 5)
        s = o.align_biwfa(p, t) if span == 2 else (o.align_endsfree(p, t) if span == 1 else o.align_end2end(p, t))
        r = res[i]
        got = cig[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes()
        assert (int(r["score"]), int(r["status"]), got) == (s, o.status(), o.cigar()[0]), (metric, mode, span, i)
    total += len(pairs)

PENS = [(1, None), (3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1]), (2, [0, 3, 2])]
short = synth.uniform_pairs(400, 100, 150, 0.0, 0.06, 911)
sp = [short.pair(i) for i in range(len(short))]
for metric, pen in PENS:
    for lanes in (4, 8, 32):
        a = pkg.WavefrontAligner(metric, pen)
        a.set_alignment_scope(True)
        a.set_lanes_per_pair(lanes)
        res, cig = a.align_batch(*pack(sp))
        check(a, res, cig, metric, pen, sp, "high", 0)
        a.close()
    for mode in ("med", "low"):
        a = pkg.WavefrontAligner(metric, pen)
        a.set_alignment_scope(True)
        a.set_memory_mode(mode)
        res, cig = a.align_batch(*pack(sp[:120]))
        check(a, res, cig, metric, pen, sp[:120], mode, 0)
        a.close()
    # The general kernel: a heuristic (WF-adaptive).
    a = pkg.WavefrontAligner(metric, pen)
    a.set_alignment_scope(True)
    a.set_heuristic(1, 10, 50, 1)
    res, cig = a.align_batch(*pack(sp[:200]))
    check(a, res, cig, metric, pen, sp[:200], "high", 0, 1, (10, 50, 1))
    a.close()
    lp = long_pairs(913 + metric, 12, 300, 900, 0.1)
    for lanes in (32, 128, 256):
        a = pkg.WavefrontAligner(metric, pen)
        a.set_alignment_scope(True)
        a.set_biwfa_lanes(lanes)
        res, cig = a.align_batch(*pack(lp), span=2)
        check(a, res, cig, metric, pen, lp, "high", 2)
        a.close()
print("checked pairs", total)
'''


def test_device_checks_build_runs_clean():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    lib = os.path.join(ROOT, "wfa2lib-rs_b200", "lib", "libwfa_b200_checked.so")
    if not os.path.exists(lib):
        pytest.skip("device-checks build not built (make -C wfa2lib-rs_b200/csrc checked)")
    env = dict(os.environ, WFA_B200_CHECKED="1")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CHILD], env=env, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "checked pairs" in r.stdout
