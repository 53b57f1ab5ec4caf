"""The oracle's med/low restatement (the piggyback backtrace) on its own
properties, beside the reference's med/low golden vectors (in
test_oracle_golden): the same score and status as high memory, a CIGAR that
spells both sequences and rescoring to that score, and med equal to low."""
import random

import pytest

import oracle as O
from test_emu_vs_oracle import PENS
from test_oracle_unit import lcg_pairs


def run(metric, pen, p, t, mode, span=0, free=None, hk=0, hp=(0, 0, 0)):
    a = O.OracleAligner(metric, pen)
    a.set_alignment_scope(True)
    a.set_memory_mode(mode)
    if hk:
        a.set_heuristic(hk, *hp)
    if span:
        a.set_alignment_free_ends(*free)
        s = a.align_endsfree(p, t)
    else:
        s = a.align_end2end(p, t)
    ops, cs, ev, eh = a.cigar()
    return s, a.status(), ops, cs


def spells(ops, p, t):
    v = h = 0
    for o in ops.decode():
        if o == "M":
            if p[v] != t[h]:
                return False
            v += 1; h += 1
        elif o == "X":
            if p[v] == t[h]:
                return False
            v += 1; h += 1
        elif o == "D":
            v += 1
        else:
            h += 1
    return (v, h) == (len(p), len(t))


@pytest.mark.parametrize("metric,pen", PENS)
def test_end2end_against_high_memory(metric, pen):
    for p, t in lcg_pairs(900 + metric, 40, 300):
        s_hi, st_hi, _, _ = run(metric, pen, p, t, "high")
        s_med, st_med, ops_med, cs_med = run(metric, pen, p, t, "med")
        s_low, st_low, ops_low, _ = run(metric, pen, p, t, "low")
        assert (s_med, st_med) == (s_hi, st_hi) == (s_low, st_low)
        assert ops_med == ops_low
        assert spells(ops_med, p, t), (p, t, ops_med)
        assert cs_med == s_med


@pytest.mark.parametrize("metric,pen", PENS)
def test_endsfree_against_high_memory(metric, pen):
    r = random.Random(metric)
    for p, t in lcg_pairs(950 + metric, 25, 200):
        free = [r.randrange(0, len(p) // 3 + 1), r.randrange(0, len(p) // 3 + 1),
                r.randrange(0, len(t) // 3 + 1), r.randrange(0, len(t) // 3 + 1)]
        s_hi, st_hi, _, _ = run(metric, pen, p, t, "high", span=1, free=free)
        s_med, st_med, ops, _ = run(metric, pen, p, t, "med", span=1, free=free)
        assert (s_med, st_med) == (s_hi, st_hi)
        assert run(metric, pen, p, t, "low", span=1, free=free)[2] == ops


@pytest.mark.parametrize("h,hp", [("wfa-adaptive", (10, 50, 1)), ("xdrop", (30, 1, 0)),
                                  ("banded-static", (-12, 12, 0))])
def test_heuristics_med_equals_low(h, hp):
    for metric, pen in [(3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1])]:
        for p, t in lcg_pairs(990 + metric, 20, 300):
            med = run(metric, pen, p, t, "med", hk=O.HEURISTICS[h], hp=hp)
            low = run(metric, pen, p, t, "low", hk=O.HEURISTICS[h], hp=hp)
            hi = run(metric, pen, p, t, "high", hk=O.HEURISTICS[h], hp=hp)
            assert med == low
            assert med[:2] == hi[:2]
