"""BiWFA device driver (host build of wfa_biwfa.cuh) against the oracle."""
import random

import pytest

import cli_format
import emu_lib
import oracle as O
from test_emu_vs_oracle import HEUR, PENS
from test_oracle_unit import lcg_pairs


def long_pairs(seed, count, lo, hi, rate):
    """Pairs long enough to recurse: substitutions and short indels."""
    r = random.Random(seed)
    out = []
    for _ in range(count):
        n = r.randrange(lo, hi)
        p = bytes(r.choice(b"ACGT") for _ in range(n))
        t, i = bytearray(), 0
        while i < n:
            x = r.random()
            if x < rate * 0.4:
                t.append(r.choice(b"ACGT")); i += 1
            elif x < rate * 0.7:
                t += bytes(r.choice(b"ACGT") for _ in range(1 + r.randrange(5)))
            elif x < rate:
                i += 1 + r.randrange(5)
            else:
                t.append(p[i]); i += 1
        out.append((p, bytes(t)))
    return out


def compare(metric, pen, pairs, compute=True, hk=0, hp=(0, 0, 0), packed=False, lanes=None, idc=0):
    res, cig = emu_lib.run_biwfa(metric, pen, pairs, compute_alignment=compute, heuristic=hk,
                                 hparams=hp, packed=packed, lanes=lanes, idc=idc)
    for i, (p, t) in enumerate(pairs):
        a = O.OracleAligner(metric, pen)
        if hk:
            a.set_heuristic(hk, *hp)
        s = a.align_biwfa(p, t) if compute else a.align_biwfa_score(p, t)
        ops = a.cigar()[0].decode() if compute else ""
        got = (int(res["score"][i]), int(res["status"][i]), cig[i] if compute else "")
        assert got == (s, a.status(), ops), (metric, pen, i, len(p), len(t), got[:2], (s, a.status()))


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("packed", [False, True])
def test_biwfa(metric, pen, packed):
    pairs = lcg_pairs(301 + metric, 10, 220) + long_pairs(303 + metric, 3, 250, 700, 0.1)
    compare(metric, pen, pairs, packed=packed)
    compare(metric, pen, pairs[:8] + pairs[-2:], compute=False, packed=packed)


@pytest.mark.parametrize("idc", [0, 1, 2])
@pytest.mark.parametrize("metric,pen", [(3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1])])
def test_biwfa_growth_idc_rings(metric, pen, idc):
    """Breakpoint searches of more than 2,048 antidiagonals keep their I/D
    rows in small rings until near the overlap scans (0); kept until the
    scans, every such search restarts with all rows kept (1); off (2).  The
    results are the same."""
    pairs = long_pairs(341 + metric, 3, 1100, 2400, 0.1)
    assert max(len(p) + len(t) for p, t in pairs) > 2100
    compare(metric, pen, pairs, packed=True, idc=idc)
    compare(metric, pen, pairs[:1], compute=False, idc=idc)


@pytest.mark.parametrize("metric,pen", [(1, None), (3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1])])
def test_biwfa_team_lanes(metric, pen):
    """The driver with 128 lanes as host threads that meet at barriers (a
    team of four warps): every collective must be reached by all of its
    lanes in the same order.  One pair that recurses (a breakpoint, base
    cases) and one short pair."""
    pairs = lcg_pairs(331 + metric, 1, 120) + long_pairs(333 + metric, 1, 420, 520, 0.1)
    compare(metric, pen, pairs, packed=True, lanes=128)
    compare(metric, pen, pairs[-1:], compute=False, lanes=128)


@pytest.mark.parametrize("h,hp", [("banded-static", (-10, 10, 0)), ("banded-adaptive", (-8, 8, 1)),
                                  ("wfa-adaptive", (10, 50, 1))])
@pytest.mark.parametrize("metric,pen", [(3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1]), (1, None)])
def test_biwfa_heuristics(metric, pen, h, hp):
    compare(metric, pen, long_pairs(311 + metric, 4, 200, 600, 0.08), hk=HEUR[h], hp=hp)


def test_biwfa_edges():
    edge = [(b"", b""), (b"A", b""), (b"", b"ACGT"), (b"A" * 300, b"C" * 300), (b"ACGT" * 60, b"ACGT" * 60)]
    for metric, pen in PENS:
        compare(metric, pen, edge)


def test_biwfa_32_lanes():
    compare(4, [0, 4, 6, 2, 24, 1], long_pairs(321, 1, 300, 400, 0.1), lanes=32)


def test_biwfa_golden_cli(golden):
    for case in golden["cases"]:
        if case["memory"] != "ultralow":
            continue
        metric = O.METRICS[case["algo"]]
        pen = [int(x) for x in case["penalties"].split(",")] if case["penalties"] else O.DEFAULT_PEN[metric]
        hk, hp = 0, (0, 0, 0)
        if case["heuristic"]:
            hk = HEUR[case["heuristic"]]
            hp = tuple(int(x) for x in case["hparams"].split(",")) + (0, 0)
        lines = []
        for p, t in case["pairs"]:
            pb, tb = p.encode(), t.encode()
            res, cig = emu_lib.run_biwfa(metric, pen, [(pb, tb)], compute_alignment=not case["score_only"],
                                         heuristic=hk, hparams=hp[:3])
            orig = (pen + [0] * 6)[:6]
            lines.append(cli_format.line(metric, orig, case["score_only"], True, res[0], cig[0], len(pb), len(tb)))
        assert lines == case["expected"], case["name"]
