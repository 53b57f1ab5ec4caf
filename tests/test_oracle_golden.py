"""The CPU oracle against the reference's own golden vectors.

tests/golden/reference_cases.json holds the align_benchmark output literals of
the reference's tests/cli_output.rs and tests/data/*.alg (extracted as text by
tests/golden/make_golden.py).  Each case is replayed through the oracle with
the same options and must print the same lines.
"""
import pytest

import oracle as O


def _cases():
    import json, os
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "reference_cases.json")) as f:
        return json.load(f)["cases"]


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_cli_golden(case):
    assert O.run_cli_case(case) == case["expected"], case["source"]


def test_issue22_zdrop_high_memory(golden):
    """tests/corrected_zdrop.rs issue_22_c_mode_follows_c: Z-drop 50,10 with a
    match reward, high memory, C mode: a valid partial alignment whose classic
    affine score is the recorded one."""
    x = golden["extra"]["issue22_zdrop_high"]
    (p, t), = x["pairs"]
    a = O.OracleAligner(3, x["penalties"])
    a.set_alignment_scope(True)
    a.set_heuristic("zdrop", *x["zdrop"])
    a.align_end2end(p.encode(), t.encode())
    ops, _, _, _ = a.cigar()
    i = j = 0
    for op in ops.decode():
        if op in "MX":
            assert i < len(p) and j < len(t) and (p[i] == t[j]) == (op == "M")
            i += 1; j += 1
        elif op == "D":
            i += 1
        else:
            j += 1
    m, x_, o, e = x["penalties"]
    score, last = 0, ""
    for op in ops.decode():
        if op == "M": score -= m
        elif op == "X": score -= x_
        else: score -= e + (0 if last == op else o)
        last = op
    assert score == x["cigar_affine_score"]
