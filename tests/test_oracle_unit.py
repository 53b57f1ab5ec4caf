"""Known-answer tests of the reference, restated against the CPU oracle.

Each test cites the reference unit test it restates; the literals are those
tests' own inputs and expected values.
"""
import random

import pytest

import oracle as O

EDIT, INDEL, LINEAR, AFFINE, AFFINE2P = 1, 0, 2, 3, 4
AFF = [0, 4, 6, 2]
AFF2P = [0, 4, 6, 2, 24, 1]
LIN = [0, 4, 2]
COMPLETED, UNREACHABLE, MAXSTEPS, PARTIAL = 5, 2, 3, 6


def cigar_str(a):
    return a.cigar()[0].decode()


def rle(ops):
    out, i = [], 0
    while i < len(ops):
        j = i
        while j < len(ops) and ops[j] == ops[i]:
            j += 1
        out.append(f"{j - i}{ops[i]}")
        i = j
    return "".join(out)


@pytest.mark.parametrize("p,t,want", [
    (b"ACGT", b"ACGT", 0), (b"ACGT", b"ACTT", 1), (b"ACT", b"ACGT", 1), (b"ACGT", b"ACT", 1),
    (b"kitten", b"sitting", 3), (b"", b"ACGT", 4), (b"ACGT", b"", 4), (b"AAAA", b"TTTT", 4),
    (b"ACGTACGTACGTACGT", b"ACGTACGTACGTACGT", 0),
])
def test_edit_scores(p, t, want):
    """src/aligner.rs:3563-3626 (test_identical_sequences .. test_longer_sequences)."""
    a = O.OracleAligner(EDIT)
    assert a.align_end2end(p, t) == want
    assert a.status() == COMPLETED


@pytest.mark.parametrize("p,t,want", [(b"ACGT", b"ACTT", 2), (b"ACGT", b"ACGT", 0), (b"ACT", b"ACGT", 1)])
def test_indel_scores(p, t, want):
    """src/aligner.rs:3629-3650."""
    assert O.OracleAligner(INDEL).align_end2end(p, t) == want


def test_reuse_aligner():
    """src/aligner.rs:3653-3659."""
    a = O.OracleAligner(EDIT)
    assert a.align_end2end(b"ACGT", b"ACTT") == 1
    assert a.align_end2end(b"AAA", b"BBB") == 3


def test_max_steps_limit():
    """src/aligner.rs:3662-3669."""
    a = O.OracleAligner(EDIT)
    a.set_max_alignment_steps(2)
    s = a.align_end2end(b"AAAA", b"TTTT")
    assert a.status() == MAXSTEPS and s <= 4


def test_edit_backtrace():
    """src/backtrace.rs:877-884: edit ACGT/ACTT -> 2M1X1M; kitten/sitting (:909-917)."""
    a = O.OracleAligner(EDIT)
    a.set_alignment_scope(True)
    assert a.align_end2end(b"ACGT", b"ACTT") == 1
    assert rle(cigar_str(a)) == "2M1X1M"
    assert a.align_end2end(b"kitten", b"sitting") == 3


@pytest.mark.parametrize("metric,pen", [(EDIT, None), (INDEL, None), (LINEAR, LIN)])
@pytest.mark.parametrize("compute", [True, False])
def test_banded_unreachable_edit_linear(metric, pen, compute):
    """src/aligner.rs:3732-3777: band [-5,5] excludes the end diagonal."""
    pattern = b"ACGTTGCAAGCT" * 10
    text = pattern[:90]
    a = O.OracleAligner(metric, pen)
    a.set_alignment_scope(compute)
    a.set_max_alignment_steps(10_000)
    a.set_heuristic("banded-static", -5, 5)
    a.align_end2end(pattern, text)
    assert a.status() == UNREACHABLE
    a.set_heuristic(None)
    a.set_alignment_scope(True)
    a.align_end2end(b"ACGTACGT", b"ACGAACGT")
    assert a.status() == COMPLETED


@pytest.mark.parametrize("compute", [True, False])
def test_banded_unreachable_affine(compute):
    """src/aligner.rs:3800-3830: give-up score 58 (C score-only)."""
    pattern = b"ACGTTGCAAGCT" * 10
    text = pattern[:90]
    a = O.OracleAligner(AFFINE, AFF)
    a.set_alignment_scope(compute)
    a.set_max_alignment_steps(10_000)
    a.set_heuristic("banded-static", -5, 5)
    assert a.align_end2end(pattern, text) == 58
    assert a.status() == UNREACHABLE
    b = O.OracleAligner(AFFINE2P, AFF2P)
    b.set_alignment_scope(compute)
    b.set_max_alignment_steps(10_000)
    b.set_heuristic("banded-static", -5, 5)
    b.align_end2end(pattern, text)
    assert b.status() == UNREACHABLE


def test_banded_end_outside_band():
    """src/aligner.rs:3833-3858."""
    p = b"GCAAGACGATTAGACTTGATAAATGCAATCATCGACTGTAAACAGACGAGCTGTCCTGGGACACTACTGACCGGATCGACTACCGCGT"
    t = b"ACAAGACACGCTCAGTGACTTGCGTCACCATCGAGCATCCGTCTTAGCAACAGGGCTGTCTGGGGCTGCCATACGACCCGCTGACCGCACGTACGGGCCT"
    for metric, pen in [(AFFINE, AFF), (AFFINE2P, AFF2P)]:
        a = O.OracleAligner(metric, pen)
        a.set_alignment_scope(True)
        a.set_heuristic("banded-static", -10, 10)
        a.align_end2end(p, t)
        assert a.status() == UNREACHABLE
        assert a.cigar()[0] == b""


def test_endsfree_begin_free_match_zero():
    """src/aligner.rs:3860-3887."""
    pairs = [(b"TTTTTACGTACGTACGT", b"ACGTACGTACGT"), (b"ACGTACGTACGT", b"GGGACGTACGTACGT"),
             (b"ACGTTCGTACGA", b"CCACGTACGTACGA")]
    a = O.OracleAligner(AFFINE, AFF)
    a.set_alignment_scope(True)
    for (p, t), (cg, sc) in zip(pairs, [("5D12M", 0), ("3I12M", 0), ("2I4M1X7M", 4)]):
        a.set_alignment_free_ends(5, 0, 3, 0)
        assert a.align_endsfree(p, t) == sc
        assert rle(cigar_str(a)) == cg
    e = O.OracleAligner(EDIT)
    for (p, t), sc in zip(pairs, [0, 0, 1]):
        e.set_alignment_free_ends(5, 0, 3, 0)
        assert e.align_endsfree(p, t) == sc


@pytest.mark.parametrize("metric,pen", [(EDIT, None), (AFFINE, AFF)])
@pytest.mark.parametrize("endsfree", [False, True])
@pytest.mark.parametrize("memory", ["high", "med", "low"])
def test_empty_sequences(metric, pen, endsfree, memory):
    """src/aligner.rs:3890-3921."""
    a = O.OracleAligner(metric, pen)
    a.set_memory_mode(memory)
    a.set_alignment_scope(True)
    if endsfree:
        a.set_alignment_free_ends(0, 0, 0, 0)
        s = a.align_endsfree(b"", b"")
    else:
        s = a.align_end2end(b"", b"")
    assert s == 0 and a.status() == COMPLETED and a.cigar()[0] == b""
    b = O.OracleAligner(metric, pen)
    assert b.align_biwfa(b"", b"") == 0 and b.cigar()[0] == b""


@pytest.mark.parametrize("memory", ["high", "med", "low"])
def test_endsfree_begin_free_seed_backtrace(memory):
    """src/aligner.rs:3924-3943."""
    a = O.OracleAligner(LINEAR, [0, 3, 3])
    a.set_memory_mode(memory)
    a.set_alignment_scope(True)
    a.set_alignment_free_ends(0, 0, 4, 11)
    a.align_endsfree(b"G", b"TCGGGACATCGAG")
    assert rle(cigar_str(a)) == "2I1M10I"


@pytest.mark.parametrize("metric,pen,p,t,want", [
    (LINEAR, LIN, b"ACGT", b"ACGT", 0), (LINEAR, LIN, b"ACGT", b"ACTT", 4), (LINEAR, LIN, b"ACT", b"ACGT", 2),
    (AFFINE, AFF, b"ACGT", b"ACGT", 0), (AFFINE, AFF, b"ACGT", b"ACTT", 4), (AFFINE, AFF, b"ACT", b"ACGT", 8),
    (AFFINE, AFF, b"AT", b"ACGT", 10),
    (AFFINE2P, AFF2P, b"ACGT", b"ACGT", 0), (AFFINE2P, AFF2P, b"ACGT", b"ACTT", 4),
    (AFFINE2P, AFF2P, b"ACT", b"ACGT", 8),
])
def test_gap_metrics(metric, pen, p, t, want):
    """src/aligner.rs:4036-4241 (linear, affine, affine2p scores)."""
    a = O.OracleAligner(metric, pen)
    a.set_alignment_scope(True)
    assert a.align_end2end(p, t) == want
    assert a.status() == COMPLETED


@pytest.mark.parametrize("metric,pen,p,t,pf,tf,want", [
    (EDIT, None, b"ACGT", b"ACGTXXXX", 0, 4, 0), (EDIT, None, b"ACGTXXXX", b"ACGT", 4, 0, 0),
    (EDIT, None, b"ACGT", b"ACTTXXXX", 0, 4, 1), (AFFINE, AFF, b"ACGT", b"ACGTXXXX", 0, 4, 0),
])
def test_endsfree_suffix(metric, pen, p, t, pf, tf, want):
    """src/aligner.rs:4247-4308."""
    a = O.OracleAligner(metric, pen)
    a.set_alignment_free_ends(0, pf, 0, tf)
    assert a.align_endsfree(p, t) == want
    assert a.status() == COMPLETED


def test_extension_basic():
    """src/aligner.rs:4345-4385."""
    a = O.OracleAligner(AFFINE, AFF)
    a.set_alignment_scope(True)
    a.set_alignment_extension()
    a.align_endsfree(b"ACGTXXXX", b"ACGTTTTT")
    ops, _, ev, eh = a.cigar()
    assert (ev, eh) == (4, 4) and a.status() == PARTIAL
    b = O.OracleAligner(AFFINE, AFF)
    b.set_alignment_scope(True)
    b.set_alignment_extension()
    assert b.align_endsfree(b"ACGT", b"ACGT") == 0 and b.status() == COMPLETED


def test_indel_score_beyond_edit_bound():
    """src/aligner.rs:4484-4496."""
    p, t = b"A" * 1500, b"C" * 1500
    a = O.OracleAligner(INDEL)
    a.set_alignment_scope(True)
    assert a.align_end2end(p, t) == 3000 and a.status() == COMPLETED
    assert rle(cigar_str(a)) == "1500I1500D"
    assert O.OracleAligner(INDEL).align_biwfa(p, t) == 3000


# --- invariants on random pairs (src/aligner.rs:4431-4482; tests/singletrack.rs) ---

def lcg_pairs(seed, count, max_len):
    r = random.Random(seed)
    out = []
    for _ in range(count):
        n = 1 + r.randrange(max_len)
        p = bytes(r.choice(b"ACGT") for _ in range(n))
        t = bytearray()
        i = 0
        while i < n:
            x = r.randrange(40)
            if x == 0:
                t.append(r.choice(b"ACGT"))
            elif x == 1:
                t += bytes(r.choice(b"ACGT") for _ in range(1 + r.randrange(12 if r.randrange(4) == 0 else 3)))
                t.append(p[i])
            elif x == 2:
                i += r.randrange(12 if r.randrange(4) == 0 else 3)
            else:
                t.append(p[i])
            i += 1
        out.append((p, bytes(t)))
    return out


def check_cigar(ops, p, t):
    i = j = 0
    for op in ops:
        if op in "MX":
            assert i < len(p) and j < len(t) and (p[i] == t[j]) == (op == "M")
            i += 1; j += 1
        elif op == "D":
            i += 1
        else:
            j += 1
    assert i == len(p) and j == len(t)


def classic(metric, pen, ops):
    if metric in (EDIT, INDEL):
        return -sum(o != "M" for o in ops)
    if metric == LINEAR:
        return -sum(pen[0] if o == "M" else pen[1] if o == "X" else pen[2] for o in ops)
    if metric == AFFINE:
        s, last = 0, ""
        for o in ops:
            s -= pen[0] if o == "M" else pen[1] if o == "X" else pen[3] + (0 if last == o else pen[2])
            last = o
        return s
    s, i = 0, 0
    while i < len(ops):
        j = i
        while j < len(ops) and ops[j] == ops[i]:
            j += 1
        L, o = j - i, ops[i]
        s -= pen[0] * L if o == "M" else pen[1] * L if o == "X" else min(pen[2] + pen[3] * L, pen[4] + pen[5] * L)
        i = j
    return s


PENS = [(EDIT, None), (INDEL, None), (LINEAR, LIN), (LINEAR, [-1, 3, 2]), (AFFINE, AFF),
        (AFFINE, [0, 1, 2, 1]), (AFFINE, [-3, 5, 3, 2]), (AFFINE2P, AFF2P), (AFFINE2P, [-1, 4, 6, 2, 24, 1])]


@pytest.mark.parametrize("metric,pen", PENS)
def test_random_invariants(metric, pen):
    """CIGAR valid, rescores to the score; BiWFA and score-only give the same score."""
    for p, t in lcg_pairs(0x51497E7A + metric, 60, 300):
        a = O.OracleAligner(metric, pen)
        a.set_alignment_scope(True)
        s = a.align_end2end(p, t)
        ops = cigar_str(a)
        check_cigar(ops, p.decode(), t.decode())
        m = 0 if pen is None else pen[0]
        want = -s if m == 0 else (-m * (len(p) + len(t)) - s) // 2
        if metric in (EDIT, INDEL):
            want = -s
        assert classic(metric, pen, ops) == want
        so = O.OracleAligner(metric, pen)
        assert so.align_end2end(p, t) == s
        bi = O.OracleAligner(metric, pen)
        assert bi.align_biwfa(p, t) == s
        check_cigar(bi.cigar()[0].decode(), p.decode(), t.decode())
        bs = O.OracleAligner(metric, pen)
        assert bs.align_biwfa_score(p, t) == s
