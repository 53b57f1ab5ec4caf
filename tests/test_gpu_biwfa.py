"""BiWFA on the GPU through the C ABI against the oracle (bit-exact)."""
import numpy as np
import pytest

import cli_format
import oracle as O
from _pkg import load
from test_emu_biwfa import long_pairs
from test_emu_vs_oracle import HEUR, PENS
from test_gpu_parity import pack
from test_oracle_unit import lcg_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return load()


def compare(pkg, metric, pen, pairs, compute=True, hk=0, hp=(0, 0, 0), packed=False, lanes=0):
    a = pkg.WavefrontAligner(metric, pen)
    a.set_alignment_scope(compute)
    if lanes:
        a.set_biwfa_lanes(lanes)
    if hk:
        a.set_heuristic(hk, *hp)
    if packed:
        from wfa_b200 import synth
        ps = synth.PairSet(*pack(pairs))
        words, pwo, two = synth.pack2bits(ps)
        res, cig = a.align_batch(np.concatenate([words, np.zeros(4, np.uint32)]), pwo, ps.p_len, two,
                                 ps.t_len, packed=True, span=2)
    else:
        seq, po, pl, to, tl = pack(pairs)
        res, cig = a.align_batch(seq, po, pl, to, tl, span=2)
    for i, (p, t) in enumerate(pairs):
        o = O.OracleAligner(metric, pen)
        if hk:
            o.set_heuristic(hk, *hp)
        s = o.align_biwfa(p, t) if compute else o.align_biwfa_score(p, t)
        ops = o.cigar()[0] if compute else b""
        r = res[i]
        got = cig[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes() if compute else b""
        assert (int(r["score"]), int(r["status"]), got) == (s, o.status(), ops), (metric, i, len(p))


@pytest.mark.parametrize("lanes", [32, 128, 256, 512])
@pytest.mark.parametrize("metric,pen", PENS)
def test_biwfa_batch(pkg, metric, pen, lanes):
    """A warp per pair, and teams of 4, 8 and 16 warps."""
    pairs = lcg_pairs(401 + metric, 30, 250) + long_pairs(403 + metric, 8, 300, 1500, 0.1)
    compare(pkg, metric, pen, pairs, lanes=lanes)
    compare(pkg, metric, pen, pairs, packed=True, lanes=lanes)
    compare(pkg, metric, pen, pairs, compute=False, lanes=lanes)


@pytest.mark.parametrize("h,hp", [("banded-static", (-10, 10, 0)), ("banded-adaptive", (-8, 8, 1)),
                                  ("wfa-adaptive", (10, 50, 1))])
def test_biwfa_heuristics(pkg, h, hp):
    for metric, pen in [(3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1])]:
        compare(pkg, metric, pen, long_pairs(411 + metric, 6, 300, 1200, 0.08), hk=HEUR[h], hp=hp)


def test_biwfa_long_affine2p(pkg):
    """Uneven long reads in the two-piece configuration (1.5-4 kbp, 5-15 %)."""
    pairs = long_pairs(421, 6, 1500, 4000, 0.15)
    compare(pkg, 4, [0, 4, 6, 2, 24, 1], pairs, packed=True)


def test_biwfa_plain_and_golden_cli(pkg, golden):
    for case in golden["cases"]:
        if case["memory"] != "ultralow":
            continue
        metric = O.METRICS[case["algo"]]
        pen = [int(x) for x in case["penalties"].split(",")] if case["penalties"] else O.DEFAULT_PEN[metric]
        a = pkg.WavefrontAligner(metric, pen)
        if case["heuristic"]:
            a.set_heuristic(case["heuristic"], *[int(x) for x in case["hparams"].split(",")])
        lines = []
        for p, t in case["pairs"]:
            pb, tb = p.encode(), t.encode()
            s = a.align_biwfa_score(pb, tb) if case["score_only"] else a.align_biwfa(pb, tb)
            c = a.cigar()
            rec = {"score": s, "status": a.status(), "end_score": 0, "end_k": 0, "end_offset": 0}
            orig = (pen + [0] * 6)[:6]
            lines.append(cli_format.line(metric, orig, case["score_only"], True, rec,
                                         "" if case["score_only"] else c.operations.decode(), len(pb), len(tb)))
        assert lines == case["expected"], case["name"]


def _batch_vs_oracle(pkg, metric, pen, ps, lanes=0):
    """A packed host-buffer BiWFA batch against the oracle's align_biwfa on
    every pair: score, status and CIGAR (hashes of the op bytes)."""
    import os
    from wfa_b200 import synth
    a = pkg.WavefrontAligner(metric, pen)
    a.set_alignment_scope(True)
    if lanes:
        a.set_biwfa_lanes(lanes)
    words, pwo, two = synth.pack2bits(ps)
    res, cig = a.align_batch(np.concatenate([words, np.zeros(4, np.uint32)]), pwo, ps.p_len, two,
                             ps.t_len, packed=True, span=2)
    a.close()
    threads = os.cpu_count() or 1
    _, sc, st, hs = O.batch(metric, pen, ps.buf.tobytes(), ps.p_off, ps.p_len, ps.t_off, ps.t_len,
                            mode=2, threads=threads)
    gh = O.hash_ops(cig, res["cigar_begin"].astype(np.int64), res["cigar_length"], threads)
    assert np.array_equal(res["score"], sc)
    assert np.array_equal(res["status"], st)
    assert np.array_equal(gh, hs)


@pytest.mark.parametrize("lanes", [32, 256])
def test_biwfa_longread_sizes(pkg, lanes):
    """Pairs of the uneven long-read batch at its long end: 16 pairs of
    8.5-20 kbp at 5-15 % edits (60 % indels), gap-affine 2-piece -- deep
    breakpoint recursions and the recovery threshold."""
    from wfa_b200 import synth
    pool = synth.config3(400, synth.SEED_BASE + 3)
    ps = pool.subset(np.where(pool.p_len >= 8000)[0][:16])
    assert len(ps) == 16 and ps.p_len.max() > 15000
    _batch_vs_oracle(pkg, 4, [0, 4, 6, 2, 24, 1], ps, lanes)


def test_biwfa_serving_long_lane(pkg):
    """Two 50 kbp pairs at 10 % edits, gap-affine: the serving mix's BiWFA lane."""
    from wfa_b200 import synth
    ps = synth.pairs_with_lengths([50000, 50000], [0.1, 0.1], 77)
    _batch_vs_oracle(pkg, 3, [0, 4, 6, 2], ps)
