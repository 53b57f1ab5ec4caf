"""The device aligner's logic (host build, one-lane warp) against the oracle.

tests/emu builds wfa2lib-rs_b200/csrc/wfa_align.cuh -- the exact source the
CUDA kernel runs -- as host C++, so every configuration here is checked on CPU
before GPU time is spent.  The GPU tests then check the real kernel the same way.
"""
import random

import numpy as np
import pytest

import cli_format
import emu_lib
import oracle as O
from test_oracle_unit import lcg_pairs

PENS = [(1, None), (0, None), (2, [0, 4, 2]), (2, [-1, 3, 2]), (3, [0, 4, 6, 2]), (3, [0, 1, 2, 1]),
        (3, [-3, 5, 3, 2]), (4, [0, 4, 6, 2, 24, 1]), (4, [-1, 4, 6, 2, 24, 1])]
HEUR = {"wfa-adaptive": 1, "xdrop": 2, "zdrop": 3, "banded-static": 4, "banded-adaptive": 5}


def oracle_run(metric, pen, p, t, compute, span, free, hk, hp, extension=False, memory="high",
               compat=0):
    a = O.OracleAligner(metric, pen)
    a.set_alignment_scope(compute)
    a.set_memory_mode(memory)
    a.set_compat(compat)
    if hk:
        a.set_heuristic(hk, *hp)
    if extension:
        a.set_alignment_extension()
        s = a.align_endsfree(p, t)
    elif span:
        a.set_alignment_free_ends(*free)
        s = a.align_endsfree(p, t)
    else:
        s = a.align_end2end(p, t)
    ops, cs, ev, eh = a.cigar()
    return s, a.status(), ops.decode() if compute else "", a.end_pos(), (cs, ev, eh)


def compare(metric, pen, pairs, compute=True, span=0, free=None, hk=0, hp=(0, 0, 0),
            extension=False, packed=False, memory="high", compat=0):
    res, cig = emu_lib.run(metric, pen, pairs, compute_alignment=compute, span=span or int(extension),
                           extension=int(extension), free=free, heuristic=hk, hparams=hp,
                           packed=packed, piggyback=memory if compute and memory != "high" else False, compat=compat)
    for i, (p, t) in enumerate(pairs):
        s, st, ops, ep, (cs, ev, eh) = oracle_run(metric, pen, p, t, compute, span, free, hk, hp,
                                                  extension, memory, compat)
        r = res[i]
        got = (int(r["score"]), int(r["status"]), cig[i] if compute else "",
               (int(r["end_score"]), int(r["end_k"]), int(r["end_offset"])))
        assert got == (s, st, ops, ep), (metric, pen, i, p, t, got, (s, st, ops, ep))
        if compute:
            assert (int(r["cigar_score"]), int(r["end_v"]), int(r["end_h"])) == (cs, ev, eh), i


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("compute", [True, False])
def test_end2end(metric, pen, compute):
    compare(metric, pen, lcg_pairs(11 + metric, 40, 250), compute=compute)


@pytest.mark.parametrize("metric,pen", PENS)
def test_endsfree(metric, pen):
    r = random.Random(metric * 7 + 1)
    pairs = lcg_pairs(23 + metric, 30, 200)
    for p, t in pairs:
        free = [r.randrange(0, len(p) // 4 + 1), r.randrange(0, len(p) // 4 + 1),
                r.randrange(0, len(t) // 4 + 1), r.randrange(0, len(t) // 4 + 1)]
        compare(metric, pen, [(p, t)], span=1, free=free)


@pytest.mark.parametrize("metric,pen", [x for x in PENS if x[0] >= 2])
def test_extension(metric, pen):
    compare(metric, pen, lcg_pairs(31 + metric, 30, 200), extension=True)


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("h,hp", [("wfa-adaptive", (10, 50, 1)), ("wfa-adaptive", (4, 5, 2)),
                                  ("xdrop", (20, 1)), ("xdrop", (20, 3)), ("zdrop", (20, 1)),
                                  ("zdrop", (15, 2)), ("banded-static", (-5, 5)),
                                  ("banded-adaptive", (-3, 3, 1))])
def test_heuristics(metric, pen, h, hp):
    if h in ("xdrop", "zdrop") and metric in (0, 1):
        pytest.skip("drops are rejected with edit/indel")
    hp = list(hp) + [0] * (3 - len(hp))
    compare(metric, pen, lcg_pairs(41 + metric, 25, 250), hk=HEUR[h], hp=hp)
    compare(metric, pen, lcg_pairs(43 + metric, 10, 150), hk=HEUR[h], hp=hp, compute=False)


@pytest.mark.parametrize("metric,pen", [x for x in PENS if x[0] >= 2])
@pytest.mark.parametrize("h,hp", [("xdrop", (30, 1, 0)), ("zdrop", (30, 1, 0))])
def test_heuristics_endsfree(metric, pen, h, hp):
    compare(metric, pen, lcg_pairs(51 + metric, 20, 200), hk=HEUR[h], hp=hp, extension=True)
    compare(metric, pen, lcg_pairs(53 + metric, 20, 200), hk=HEUR[h], hp=hp, span=1, free=[5, 5, 5, 5])


@pytest.mark.parametrize("packed", [False, True])
def test_packed_and_edges(packed):
    edge = [(b"", b""), (b"A", b""), (b"", b"ACGT"), (b"A", b"C"), (b"A", b"A"),
            (b"ACGTACGTACGTACGTACGTAC", b"ACGTACGTACGTACGTACGTAC"), (b"ACGT" * 40, b"ACGT" * 40),
            (b"AAAAAAAA", b"CCCCCCCC"), (b"ACGTTTTTTTTTTACGT", b"ACGTACGT")]
    for metric, pen in PENS:
        compare(metric, pen, edge, packed=packed)


# Med/low memory with an alignment: the piggyback backtrace.
@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("memory", ["med", "low"])
def test_piggyback_end2end(metric, pen, memory):
    compare(metric, pen, lcg_pairs(61 + metric, 30, 250), memory=memory)


@pytest.mark.parametrize("metric,pen", PENS)
def test_piggyback_endsfree(metric, pen):
    r = random.Random(metric * 11 + 3)
    for p, t in lcg_pairs(67 + metric, 20, 200):
        free = [r.randrange(0, len(p) // 3 + 1), r.randrange(0, len(p) // 3 + 1),
                r.randrange(0, len(t) // 3 + 1), r.randrange(0, len(t) // 3 + 1)]
        compare(metric, pen, [(p, t)], span=1, free=free, memory="med")


@pytest.mark.parametrize("metric,pen", [x for x in PENS if x[0] >= 2])
def test_piggyback_extension(metric, pen):
    compare(metric, pen, lcg_pairs(71 + metric, 20, 200), extension=True, memory="low")


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("h,hp", [("wfa-adaptive", (10, 50, 1)), ("xdrop", (20, 1)),
                                  ("banded-static", (-5, 5)), ("banded-adaptive", (-3, 3, 1))])
def test_piggyback_heuristics(metric, pen, h, hp):
    if h in ("xdrop", "zdrop") and metric in (0, 1):
        pytest.skip("drops are rejected with edit/indel")
    hp = list(hp) + [0] * (3 - len(hp))
    compare(metric, pen, lcg_pairs(73 + metric, 20, 250), hk=HEUR[h], hp=hp, memory="med")


def test_piggyback_edges():
    edge = [(b"", b""), (b"A", b""), (b"", b"ACGT"), (b"A", b"C"), (b"A", b"A"),
            (b"ACGT" * 40, b"ACGT" * 40), (b"AAAAAAAA", b"CCCCCCCC"), (b"ACGTTTTTTTTTTACGT", b"ACGTACGT")]
    for metric, pen in PENS:
        compare(metric, pen, edge, memory="med")
        for p, t in edge:  # free ends within the lengths, as the aligner requires
            free = [min(2, len(p)), min(1, len(p)), min(2, len(t)), min(1, len(t))]
            compare(metric, pen, [(p, t)], span=1, free=free, memory="low")


# Compat::Corrected: ends-free with a match reward (candidate, diagonal and
# dominance pruning) and Z-drop ends.
CORR_PENS = [(2, [-1, 3, 2]), (2, [-3, 4, 5]), (3, [-3, 5, 3, 2]), (3, [-5, 4, 0, 8]),
             (4, [-1, 4, 6, 2, 24, 1]), (4, [-2, 4, 0, 6, 10, 2])]


@pytest.mark.parametrize("metric,pen", CORR_PENS)
@pytest.mark.parametrize("memory", ["high", "med"])
def test_corrected_endsfree(metric, pen, memory):
    r = random.Random(metric * 5 + len(memory))
    for p, t in lcg_pairs(81 + metric, 24, 160):
        n, m = len(p), len(t)
        free = [r.choice([0, n, r.randrange(n + 1)]), r.choice([0, n, r.randrange(n + 1)]),
                r.choice([0, m, r.randrange(m + 1)]), r.choice([0, m, r.randrange(m + 1)])]
        compare(metric, pen, [(p, t)], span=1, free=free, memory=memory, compat=1)
        compare(metric, pen, [(p, t)], compute=False, span=1, free=free, compat=1)


@pytest.mark.parametrize("metric,pen", CORR_PENS)
def test_corrected_dominance(metric, pen):
    """Small begin-free tolerances: the dominance pruning is active."""
    for i, (p, t) in enumerate(lcg_pairs(87 + metric, 30, 200)):
        b = 1 + i % 5
        e = 0 if i % 2 else min(16, len(p), len(t))
        free = [min(b, len(p)), min(e, len(p)), min(b, len(t)), min(e, len(t))]
        compare(metric, pen, [(p, t)], span=1, free=free, memory=["high", "low"][i % 2], compat=1)


@pytest.mark.parametrize("metric,pen", CORR_PENS)
def test_corrected_extension_and_heuristics(metric, pen):
    pairs = lcg_pairs(91 + metric, 20, 200)
    compare(metric, pen, pairs, extension=True, compat=1)
    compare(metric, pen, pairs, extension=True, memory="med", compat=1)
    for hk, hp in ((4, (-20, 20, 0)), (2, (30, 1, 0)), (3, (30, 1, 0)), (1, (10, 50, 1))):
        compare(metric, pen, pairs, hk=hk, hp=hp, compat=1)
        compare(metric, pen, pairs, hk=hk, hp=hp, memory="med", compat=1)
        compare(metric, pen, pairs[:8], span=1, free=[5, 5, 5, 5], hk=hk, hp=hp, compat=1)


def test_golden_cli_cases(golden):
    """The reference's CLI golden lines, reproduced by the device logic."""
    checked = 0
    for case in golden["cases"]:
        if case["memory"] not in ("high", "med", "low"):
            continue
        metric = O.METRICS[case["algo"]]
        pen = [int(x) for x in case["penalties"].split(",")] if case["penalties"] else O.DEFAULT_PEN[metric]
        so = case["score_only"]
        span_s = case["span"]
        hk, hp = 0, (0, 0, 0)
        if case["heuristic"]:
            hk = HEUR[case["heuristic"]]
            hp = [int(x) for x in case["hparams"].split(",")] + [0, 0]
        lines = []
        for p, t in case["pairs"]:
            pb, tb = p.encode(), t.encode()
            span, ext, free = 0, 0, None
            if span_s in ("extension", "extend"):
                span, ext = 1, 1
            elif span_s != "global":
                fr = [float(x) for x in span_s.split(",")[1:]]
                free = [O.nominal_prop(len(pb), fr[0]), O.nominal_prop(len(pb), fr[1]),
                        O.nominal_prop(len(tb), fr[2]), O.nominal_prop(len(tb), fr[3])]
                span = 1
            res, cig = emu_lib.run(metric, pen, [(pb, tb)], compute_alignment=not so, span=span,
                                   extension=ext, free=free, heuristic=hk, hparams=hp[:3],
                                   piggyback=case["memory"] if not so and case["memory"] != "high" else False,
                                   compat=int(case.get("no_c_compat", False)))
            orig = (pen + [0] * 6)[:6]
            lines.append(cli_format.line(metric, orig, so, False, res[0], cig[0], len(pb), len(tb),
                                         case.get("no_c_compat", False)))
        assert lines == case["expected"], case["name"]
        checked += 1
    assert checked >= 20


# Med/low on the configurations where the kernels' picks depend on values a
# later step changes (a heuristic emptying I/D of the same score; C-mode
# Z-drop ends read on a dead cell), and with the backtrace buffer compacted
# every few scores under a tiny limit: the oracle, which never compacts,
# must still agree on every pair (compaction keeps every live chain whole).
@pytest.mark.parametrize("memory", ["med", "low"])
def test_piggyback_picks_and_compaction(memory):
    import random
    rng = random.Random(4242)
    pairs = []
    for _ in range(30):
        n = rng.randint(40, 400)
        p = bytes(rng.choice(b"ACGT") for _ in range(n))
        t = bytearray()
        for c in p:
            u = rng.random()
            if u < 0.05: t += bytes([rng.choice(b"ACGT")])
            elif u < 0.10: t += bytes([rng.choice(b"ACGT"), c])
            elif u < 0.15: pass
            else: t.append(c)
        pairs.append((p, bytes(t)))
    cases = [(3, [-3, 5, 3, 2], 1, 5, (-8, 8, 1)), (4, [-1, 4, 6, 2, 24, 1], 0, 3, (20, 1, 0)),
             (4, [-1, 4, 6, 2, 24, 1], 1, 5, (-8, 8, 1)), (3, [0, 4, 6, 2], 0, 0, (0, 0, 0)),
             (1, None, 0, 0, (0, 0, 0)), (2, [0, 4, 2], 1, 1, (10, 50, 1))]
    for metric, pen, span, hk, hp in cases:
        for probe, limit in ((6000, 256 << 20), (3, 64)):
            for p, t in pairs:
                free = [len(p) // 5, len(p) // 5, len(t) // 5, len(t) // 5] if span else None
                res, cig = emu_lib.run(metric, pen, [(p, t)], span=span, free=free, heuristic=hk,
                                       hparams=hp, piggyback=memory, bt_limit=limit, bt_probe=probe,
                                       bt_cap=1 << 16)
                s, st, ops, ep, cg = oracle_run(metric, pen, p, t, True, span, free, hk, list(hp),
                                                memory=memory)
                assert (int(res["score"][0]), int(res["status"][0]), cig[0]) == (s, st, ops), \
                    (metric, pen, span, hk, probe, len(p))
