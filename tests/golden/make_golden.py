"""Generate tests/golden/reference_cases.json from the reference's own tests.

The wfa2lib-rs crate cannot be built here (no Rust toolchain), so its golden
vectors are taken from its test files *as text*: the align_benchmark output
literals of tests/cli_output.rs, the C-driver outputs under tests/data/, and
the Z-drop expectation of tests/corrected_zdrop.rs.  Every sequence and every
expected line below is read from those files; nothing is typed in by hand.

Run from the repository root:  python tests/golden/make_golden.py REF_ROOT
where REF_ROOT is a checkout of the reference crate (or set WFA_REFERENCE_ROOT).
The committed JSON is what the tests read; the reference tree is not needed
at test time.
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WFA_REFERENCE_ROOT")
if not REF:
    sys.exit("usage: make_golden.py REF_ROOT (or set WFA_REFERENCE_ROOT)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def rust_strings(text):
    """String literals of a Rust snippet, escapes resolved."""
    out = []
    for m in re.finditer(r'"((?:[^"\\]|\\.)*)"', text):
        out.append(m.group(1).encode().decode("unicode_escape"))
    return out


def fn_body(src, name):
    i = src.index("fn " + name + "(")
    j = src.index("\n}\n", i)
    return src[i:j], src[:i].count("\n") + 1, src[:j].count("\n") + 1


def const_pairs(src, name):
    i = src.index("const " + name)
    j = src.index("];", i)
    s = rust_strings(src[i:j])
    return [s[k:k + 2] for k in range(0, len(s), 2)]


def seq_file(rel):
    lines = read(rel).splitlines()
    pairs = []
    for a, b in zip(lines[0::2], lines[1::2]):
        pairs.append([a.lstrip(">"), b.lstrip("<")])
    return pairs


cases = []


def add(name, src, pairs, expected, algo="gap-affine-wfa", penalties=None, span="global",
        score_only=False, memory="high", heuristic=None, hparams=None, no_c_compat=False):
    case = dict(name=name, source=src, algo=algo, penalties=penalties, span=span,
                score_only=score_only, memory=memory, heuristic=heuristic,
                hparams=hparams, pairs=pairs, expected=expected)
    if no_c_compat:  # the driver's --no-c-compat (Compat::Corrected)
        case["no_c_compat"] = True
    cases.append(case)


cli = read("tests/cli_output.rs")
CLI = "tests/cli_output.rs"

# --- empty_cigar_prints_minus_one_and_dash ---------------------------------
body, a, b = fn_body(cli, "empty_cigar_prints_minus_one_and_dash")
unit = re.search(r'let pattern = "([ACGT]+)"\.repeat\((\d+)\);', body)
cut = int(re.search(r"&pattern\[\.\.(\d+)\]", body).group(1))
pattern = unit.group(1) * int(unit.group(2))
band_pair = [[pattern, pattern[:cut]]]
algos = re.findall(r'"((?:edit|gap-linear|gap-affine|gap-affine2p)-wfa)"', body)
band = re.search(r'--wfa-heuristic-parameters=([-\d,]+)', body).group(1)
exp = re.search(r'assert_eq!\(lines, \["([^"]*)"\]', body).group(1).encode().decode("unicode_escape")
for algo in algos:
    add("unreachable_band_" + algo, f"{CLI}:{a}-{b}", band_pair, [exp], algo=algo,
        heuristic="banded-static", hparams=band)

# --- completed_alignment_prints_score_and_cigar / score_only -------------
body, a, b = fn_body(cli, "completed_alignment_prints_score_and_cigar")
s = rust_strings(body)
seqs = [x for x in s if re.fullmatch(r"[ACGT]+", x)]
add("completed", f"{CLI}:{a}-{b}", [seqs[0:2], seqs[2:4]], s[-2:])
body, a, b = fn_body(cli, "score_only_prints_dash_cigar")
s = rust_strings(body)
seqs = [x for x in s if re.fullmatch(r"[ACGT]+", x)]
add("score_only", f"{CLI}:{a}-{b}", [seqs[0:2]], s[-1:], score_only=True)

# --- wfa_span_matches_c ----------------------------------------------------
span_pairs = const_pairs(cli, "SPAN_PAIRS")
body, a, b = fn_body(cli, "wfa_span_matches_c")
for m in re.finditer(r'span\("(\w+)", "([^"]+)", (true|false)\),\s*\[([^\]]*)\]', body):
    add("span_" + m.group(1), f"{CLI}:{a}-{b}", span_pairs, rust_strings(m.group(4)),
        span=m.group(2), score_only=m.group(3) == "true")

# --- ends_free_begin_gaps_match_c --------------------------------------------
body, a, b = fn_body(cli, "ends_free_begin_gaps_match_c")
ps = rust_strings(body[: body.index("];")])
bf_pairs = [ps[i:i + 2] for i in range(0, len(ps), 2)]
span = re.search(r'"--wfa-span=([^"]+)"', body).group(1)
mpen = re.search(r'"--affine-penalties=([-\d,]+)"', body).group(1)
runs = list(re.finditer(r'run\(\s*"(\w+)",.*?\);\s*assert_eq!\(lines, \[([^\]]*)\]\)', body, re.S))
for m in runs:
    call = m.group(0)
    add("endsfree_begin_" + m.group(1), f"{CLI}:{a}-{b}", bf_pairs, rust_strings(m.group(2)),
        span=span, score_only="--wfa-score-only" in call,
        penalties=mpen if ", m," in call or "m," in call.split("&[")[1] else None)

# --- xdrop_zdrop_match_c ---------------------------------------------------
drop_pairs = const_pairs(cli, "DROP_PAIRS")
body, a, b = fn_body(cli, "xdrop_zdrop_match_c")
full = rust_strings(body[body.index("let full = ["): body.index("];", body.index("let full = ["))])
for m in re.finditer(r'drop\("(\w+)", "(\w+)", "([\d,]+)", &\[\]\),\s*full', body):
    add("drop_" + m.group(1), f"{CLI}:{a}-{b}", drop_pairs, full, heuristic=m.group(2),
        hparams=m.group(3))
m = re.search(r'drop\("(zd_ext)", "(\w+)", "([\d,]+)", &\["--wfa-span=extension"\]\),\s*\["([^"]*)", full\[1\]\]', body)
add("drop_" + m.group(1), f"{CLI}:{a}-{b}", drop_pairs,
    [m.group(4).encode().decode("unicode_escape"), full[1]], heuristic=m.group(2),
    hparams=m.group(3), span="extension")
mpen2 = re.search(r'"--affine-penalties=([-\d,]+)", "--wfa-score-only"', body).group(1)
for m in re.finditer(r'drop\("(\w+_s)", "(\w+)", "([\d,]+)", &m\), \[([^\]]*)\]', body):
    add("drop_" + m.group(1), f"{CLI}:{a}-{b}", drop_pairs, rust_strings(m.group(4)),
        heuristic=m.group(2), hparams=m.group(3), penalties=mpen2, score_only=True)

# --- biwfa_heuristics_match_c ----------------------------------------------
(p1, t1), (p2, t2) = drop_pairs
bi_pairs = [[p1 + p2 + p1, t1 + t2 + t1], [p2 + p1 + p2, t2 + t1 + t2]]
body, a, b = fn_body(cli, "biwfa_heuristics_match_c")
fullbi = re.search(r'let full = "([^"]+)";', body).group(1)
first = rust_strings(re.search(r'let banded = \[(.*?)\];', body, re.S).group(1))[0]
pre = re.search(r'format!\("([^"]*)\{full\}"\)', body).group(1).encode().decode("unicode_escape")
banded = [first.encode().decode("unicode_escape"), pre + fullbi]
for m in re.finditer(r'biwfa\("(\w+)", "([\w-]+)", "([-\d,]+)", &\[\]\)', body):
    add("biwfa_" + m.group(1), f"{CLI}:{a}-{b}", bi_pairs, banded, memory="ultralow",
        heuristic=m.group(2), hparams=m.group(3))

# --- biwfa_match_reward_tie_breaks_match_c -----------------------------------
body, a, b = fn_body(cli, "biwfa_match_reward_tie_breaks_match_c")
s = rust_strings(body)
seqs = [x for x in s if re.fullmatch(r"[ACGT]+", x)]
pen = re.search(r'"--affine-penalties=([-\d,]+)"', body).group(1)
add("biwfa_tie", f"{CLI}:{a}-{b}", [seqs[0:2]], s[-1:], penalties=pen, memory="ultralow")

# --- memory_med_low_match_c --------------------------------------------------
body, a, b = fn_body(cli, "memory_med_low_match_c")
hp = re.search(r'"--wfa-heuristic-parameters=([\d,]+)"', body).group(1)
xm_pairs = seq_file("tests/data/xdrop_med.seq")
for mem, alg in re.findall(r'\("(med|low|high)", "([\w.]+)"\)', body):
    add("xdrop_med_" + mem, f"{CLI}:{a}-{b} + tests/data/{alg}", xm_pairs,
        read("tests/data/" + alg).splitlines(), memory=mem, heuristic="xdrop", hparams=hp)

# --- unreachable_score_only_corrected_prints_minus_one (C-mode lines) -------
body, a, b = fn_body(cli, "unreachable_score_only_corrected_prints_minus_one")
pen = re.search(r'"--affine-penalties=([-\d,]+)"', body).group(1)
hp = re.search(r'"--wfa-heuristic-parameters=([\d,]+)"', body).group(1)
exp = re.search(r'assert_eq!\(run_file\("issue23_unreachable\.seq", &args\), "([^"]*)"\);', body)
add("issue23_unreachable", f"{CLI}:{a}-{b}", seq_file("tests/data/issue23_unreachable.seq"),
    [exp.group(1).encode().decode("unicode_escape").rstrip("\n")], penalties=pen,
    heuristic="xdrop", hparams=hp, score_only=True)
exp = re.search(r'args\.push\("--no-c-compat"\);\s*assert_eq!\(run_file\("issue23_unreachable\.seq", '
                r'&args\), "([^"]*)"\);', body)
add("issue23_unreachable_corrected", f"{CLI}:{a}-{b}", seq_file("tests/data/issue23_unreachable.seq"),
    [exp.group(1).encode().decode("unicode_escape").rstrip("\n")], penalties=pen,
    heuristic="xdrop", hparams=hp, score_only=True, no_c_compat=True)
m = re.search(r'assert_eq!\(run\("unreachable_bi", &pair, &args\), \["([^"]*)"\]\);', body)
add("unreachable_biwfa_score", f"{CLI}:{a}-{b}", band_pair,
    [m.group(1).encode().decode("unicode_escape")], penalties=pen, memory="ultralow",
    heuristic="banded-static", hparams=band, score_only=True)

# --- corrected_zdrop.rs: issue_22_c_mode_follows_c (high memory) -------------
zd = read("tests/corrected_zdrop.rs")
body, a, b = fn_body(zd, "issue_22_c_mode_follows_c")
hi_score = int(re.search(r"high\.score_gap_affine\(&PEN\), (\d+)\)", body).group(1))
pen = re.search(r"match_: (-?\d+),\s*mismatch: (\d+),\s*gap_opening: (\d+),\s*gap_extension: (\d+)", zd)
zp = re.search(r"zdrop: (\d+),\s*steps_between_cutoffs: (\d+)", zd)
extra = dict(
    issue22_zdrop_high=dict(
        source=f"tests/corrected_zdrop.rs:{a}-{b}",
        penalties=[int(x) for x in pen.groups()],
        zdrop=[int(x) for x in zp.groups()],
        pairs=seq_file("tests/data/issue22_zdrop.seq"),
        cigar_affine_score=-hi_score if hi_score < 0 else hi_score,
    ),
    issue21_xdrop=dict(source="tests/xdrop_steps.rs", pairs=seq_file("tests/data/issue21_xdrop.seq")),
)

with open(OUT, "w") as f:
    json.dump(dict(generated_from="wfa2lib-rs tests (read as text)", cases=cases, extra=extra), f,
              indent=1)
print(f"wrote {len(cases)} CLI cases to {OUT}")
