"""Compat::Corrected in the oracle (src/aligner.rs:53-94, 1104-1345).

Pinned by the reference's own tests: the literal cases of
tests/corrected_endsfree.rs (issue 37's corrected CIGAR and score, issue
38's all-gap C result against the optimum), its property -- the corrected
ends-free score and the CIGAR's ends-free penalty both equal the optimum a
dynamic program finds, in score-only and every memory mode -- on seeded
random pairs, and tests/corrected_zdrop.rs (every memory mode gives the same
valid partial alignment)."""
import json
import os
import random

import pytest

import oracle as O

INDEL, EDIT, LINEAR, AFFINE, AFFINE2P = 0, 1, 2, 3, 4
HERE = os.path.dirname(os.path.abspath(__file__))


def gap_cost(pen, l):
    return min(pen["o1"] + l * pen["e1"], pen["o2"] + l * pen["e2"])


def dp_optimum(pen, p, t, ends):
    """Optimal ends-free penalty (lower is better; matches cost `match`,
    usually a reward): an alignment starts at (v, 0) with v <= pattern
    begin-free or (0, h) with h <= text begin-free, and ends at (v, |T|) with
    |P| - v <= pattern end-free or (|P|, h) with |T| - h <= text end-free."""
    inf = 1 << 60
    pb, pe, tb, te = ends
    n, m = len(p), len(t)
    pieces = [(pen["o1"], pen["e1"]), (pen["o2"], pen["e2"])]
    H = [[inf] * (m + 1) for _ in range(n + 1)]
    ins = [[[inf, inf] for _ in range(m + 1)] for _ in range(n + 1)]
    dele = [[[inf, inf] for _ in range(m + 1)] for _ in range(n + 1)]
    for v in range(n + 1):
        for j in range(m + 1):
            best = 0 if (j == 0 and v <= pb) or (v == 0 and j <= tb) else inf
            if v and j and H[v - 1][j - 1] < inf:
                best = min(best, H[v - 1][j - 1] + (pen["match"] if p[v - 1] == t[j - 1] else pen["mismatch"]))
            for i, (o, e) in enumerate(pieces):
                if j:
                    ins[v][j][i] = min(H[v][j - 1] + o + e, ins[v][j - 1][i] + e)
                    best = min(best, ins[v][j][i])
                if v:
                    dele[v][j][i] = min(H[v - 1][j] + o + e, dele[v - 1][j][i] + e)
                    best = min(best, dele[v][j][i])
            H[v][j] = best
    out = min([H[v][m] for v in range(n + 1) if n - v <= pe] + [H[n][j] for j in range(m + 1) if m - j <= te])
    return out


def cigar_penalty(pen, ops, ends):
    """Ends-free penalty of a CIGAR: a leading or trailing gap run is free up
    to its free-end limit, the rest of it is charged as a gap."""
    pb, pe, tb, te = ends
    runs = []
    for op in ops:
        if runs and runs[-1][0] == op:
            runs[-1][1] += 1
        else:
            runs.append([op, 1])
    total = 0
    for i, (op, l) in enumerate(runs):
        charged = l
        if i == 0:
            charged -= min(charged, {"D": pb, "I": tb}.get(op, 0))
        if i == len(runs) - 1:
            charged -= min(charged, {"D": pe, "I": te}.get(op, 0))
        if op == "M":
            total += l * pen["match"]
        elif op == "X":
            total += l * pen["mismatch"]
        elif charged > 0:
            total += gap_cost(pen, charged)
    return total


def valid(ops, p, t):
    i = j = 0
    for op in ops:
        if op in "MX":
            if i >= len(p) or j >= len(t) or (p[i] == t[j]) != (op == "M"):
                return False
            i += 1
            j += 1
        elif op == "D":
            i += 1
        else:
            j += 1
    return i == len(p) and j == len(t)


def penalties(kind, pen):
    """(metric, oracle penalties) for kind 0 linear, 1 affine, 2 affine2p."""
    if kind == 0:
        return LINEAR, [pen["match"], pen["mismatch"], pen["e1"]]
    if kind == 1:
        return AFFINE, [pen["match"], pen["mismatch"], pen["o1"], pen["e1"]]
    return AFFINE2P, [pen["match"], pen["mismatch"], pen["o1"], pen["e1"], pen["o2"], pen["e2"]]


def wf_to_sw(match, n, m, w):
    a = -match * (n + m) - w
    return a // 2 if a >= 0 else -((-a) // 2)


def align(metric, opens, p, t, ends, memory="high", cigar=True, compat="corrected"):
    a = O.OracleAligner(metric, opens)
    a.set_compat(compat)
    a.set_memory_mode(memory)
    a.set_alignment_scope(cigar)
    a.set_alignment_free_ends(*ends)
    w = a.align_endsfree(p.encode(), t.encode())
    match = opens[0] if opens else 0
    pen = -wf_to_sw(match, len(p), len(t), w) if match < 0 else w
    return pen, a.cigar()[0].decode() if cigar else None


def check(kind, pen, p, t, ends):
    metric, opens = penalties(kind, pen)
    want = dp_optimum(pen, p, t, ends)
    got, _ = align(metric, opens, p, t, ends, cigar=False)
    assert got == want, ("score-only", kind, pen, p, t, ends)
    for memory in ("high", "med", "low"):
        got, ops = align(metric, opens, p, t, ends, memory)
        assert got == want, (memory, kind, pen, p, t, ends)
        assert valid(ops, p, t), (memory, ops)
        assert cigar_penalty(pen, ops, ends) == want, (memory, ops, kind, pen, p, t, ends)


def affine(match, mismatch, o, e):
    return dict(match=match, mismatch=mismatch, o1=o, e1=e, o2=o, e2=e)


def test_issue_37_repeat_shift():
    """tests/corrected_endsfree.rs issue_37_repeat_shift"""
    pen = affine(-5, 4, 0, 8)
    p, t, ends = "ACGTACGTACGT", "ACGACGTACGT", (12, 12, 11, 11)
    assert dp_optimum(pen, p, t, ends) == -47
    _, c_ops = align(AFFINE, [-5, 4, 0, 8], p, t, ends, compat="c")
    assert c_ops == "IIIMMMMMMMMDDDD"
    score, ops = align(AFFINE, [-5, 4, 0, 8], p, t, ends)
    assert score == -47 and ops == "MMMDMMMMMMMM"
    check(1, pen, p, t, ends)


def test_issue_38_whole_length_free_ends():
    """tests/corrected_endsfree.rs issue_38_whole_length_free_ends"""
    pen = affine(-5, 4, 0, 8)
    p = "AAGAAGCACCGGCTAACTCCGTGCCAGCAGCCGCGGT"
    t = "AGTCGTGACTCTTTTTGCATGTACCTTATGAATAAGGACCGGCTAATTCCG"
    ends = (len(p), len(p), len(t), len(t))
    _, c_ops = align(AFFINE, [-5, 4, 0, 8], p, t, ends, compat="c")
    assert set(c_ops) <= set("ID")
    assert dp_optimum(pen, p, t, ends) == -78
    check(1, pen, p, t, ends)
    check(1, pen, "CAGA", "GGGA", (4, 4, 4, 4))


def test_match_zero_identical_to_c():
    r = random.Random(7)
    for _ in range(150):
        kind = r.randrange(3)
        pen = dict(match=0, mismatch=1 + r.randrange(6), o1=r.randrange(6), e1=1 + r.randrange(4),
                   o2=r.randrange(12), e2=1 + r.randrange(2))
        if kind < 2:
            pen.update(o2=pen["o1"], e2=pen["e1"])
        if kind == 0:
            pen.update(o1=0, o2=0)
        metric, opens = penalties(kind, pen)
        p = "".join(r.choice("ACGT") for _ in range(r.randrange(16)))
        t = "".join(r.choice("ACGT") for _ in range(r.randrange(16)))
        ends = (r.randrange(len(p) + 1), r.randrange(len(p) + 1), r.randrange(len(t) + 1),
                r.randrange(len(t) + 1))
        for memory in ("high", "med"):
            assert align(metric, opens, p, t, ends, memory, compat="c") == \
                align(metric, opens, p, t, ends, memory)


def random_pen(r, kind, match):
    if kind == 0:
        x = 1 + r.randrange(8)
        return dict(match=match, mismatch=1 + r.randrange(8), o1=0, e1=x, o2=0, e2=x)
    if kind == 1:
        return affine(match, 1 + r.randrange(8), r.randrange(8), 1 + r.randrange(8))
    o1, e1 = r.randrange(6), 2 + r.randrange(6)
    return dict(match=match, mismatch=1 + r.randrange(8), o1=o1, e1=e1, o2=o1 + 2 + r.randrange(10), e2=1)


def test_random_against_dp():
    r = random.Random(42)
    for it in range(600):
        kind = r.randrange(3)
        pen = random_pen(r, kind, -1 - r.randrange(6))
        alpha = "AC" if it % 2 == 0 else "ACGT"
        p = "".join(r.choice(alpha) for _ in range(r.randrange(20)))
        t = "".join(r.choice(alpha) for _ in range(r.randrange(20)))
        if it % 3 == 0:
            base = "".join(r.choice(alpha) for _ in range(r.randrange(6)))
            p, t = base * (1 + r.randrange(4)), base * (1 + r.randrange(4))
            if t:
                i = r.randrange(len(t))
                t = t[:i] + t[i + 1:]
        n, m = len(p), len(t)
        ends = [(n, n, m, m), (0, n, 0, m)][it % 4] if it % 4 < 2 else \
            (r.randrange(n + 1), r.randrange(n + 1), r.randrange(m + 1), r.randrange(m + 1))
        check(kind, pen, p, t, ends)


def test_small_begin_free_dominance():
    """Begin-free tolerance of 1-5 bases (dominance pruning active up to 4,
    and always with gap-linear) on mutants of a shared core."""
    r = random.Random(11)
    for it in range(60):
        kind = r.randrange(3)
        pen = [dict(match=-5, mismatch=4, o1=0, e1=8, o2=0, e2=8), affine(-5, 4, r.randrange(6), 8),
               dict(match=-5, mismatch=4, o1=0, e1=8, o2=10, e2=4)][kind]
        core = [r.choice("ACGT") for _ in range(80)]
        rate = 10 + r.randrange(40)

        def mutant():
            s = []
            for c in core:
                x = r.randrange(rate)
                if x == 0:
                    s.append(r.choice("ACGT"))
                elif x == 2:
                    s += [c, r.choice("ACGT")]
                elif x != 1:
                    s.append(c)
            k = r.randrange(4)
            if k == 0:
                s = s[1 + r.randrange(3):]
            elif k == 1:
                s = [r.choice("ACGT") for _ in range(1 + r.randrange(3))] + s
            return "".join(s)
        p, t = mutant(), mutant()
        b = 1 + it % 5
        e = 0 if it % 2 == 0 else 16
        check(kind, pen, p, t, (b, e, b, e))


def test_cli_no_c_compat_unreachable_score_only(golden):
    """tests/cli_output.rs unreachable_score_only_corrected_prints_minus_one"""
    case = next(c for c in golden["cases"] if c["name"] == "issue23_unreachable")
    c_mode = dict(case, score_only=True)
    assert O.run_cli_case(c_mode) == ["-113\t-"]
    assert O.run_cli_case(dict(c_mode, no_c_compat=True)) == ["-1\t-"]


def test_issue_22_corrected_modes_agree(golden):
    """tests/corrected_zdrop.rs issue_22_corrected_modes_agree: Z-drop 50,10
    with a match reward -- in Corrected mode every memory mode backtraces the
    best cell at its own score and gives the same valid partial alignment."""
    x = golden["extra"]["issue22_zdrop_high"]
    (p, t), = x["pairs"]
    m_, x_, o, e = x["penalties"]
    out = {}
    for memory in ("high", "med", "low"):
        a = O.OracleAligner(AFFINE, x["penalties"])
        a.set_compat("corrected")
        a.set_memory_mode(memory)
        a.set_alignment_scope(True)
        a.set_heuristic("zdrop", *x["zdrop"])
        a.align_end2end(p.encode(), t.encode())
        ops = a.cigar()[0].decode()
        i = j = 0
        for op in ops:
            if op in "MX":
                assert i < len(p) and j < len(t) and (p[i] == t[j]) == (op == "M"), memory
                i += 1
                j += 1
            elif op == "D":
                i += 1
            else:
                j += 1
        score, last = 0, ""
        for op in ops:
            score -= m_ if op == "M" else x_ if op == "X" else e + (0 if last == op else o)
            last = op
        out[memory] = score
    assert out["high"] == x["cigar_affine_score"]
    assert out["med"] == out["high"] and out["low"] == out["high"]
