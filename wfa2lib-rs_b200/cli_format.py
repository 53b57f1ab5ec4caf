"""align_benchmark's output line from an alignment result.

The per-pair output of the reference's driver (src/bin/align_benchmark.rs:
466-504, compute_output_score, and :630-672, the C-compatible line): the
score column is -(CIGAR penalty) in CIGAR mode, the negated (or, with a
match reward, Eizenga-corrected) WFA score in score-only mode, INT_MIN for a
failed BiWFA score-only run and -1 with an empty CIGAR; the CIGAR column is
the run-length string (Cigar::to_string_rle) or "-".  `r` is a mapping with
the fields of wfa_result_t (score, status, end_score, end_k, end_offset).
With `corrected` (the driver's --no-c-compat), a score-only run with no
alignment behind it prints -1 (:396-405, :641-652).
"""
INT_MIN = -2**31
NULL = -(2**30)


def _wrap(x):
    return (x + 2**31) % 2**32 - 2**31


def rle(ops):
    out, i = [], 0
    while i < len(ops):
        j = i
        while j < len(ops) and ops[j] == ops[i]:
            j += 1
        out.append(f"{j - i}{ops[i]}")
        i = j
    return "".join(out)


def classic_score(metric, orig, ops):
    if metric in (0, 1):
        return sum(o != "M" for o in ops)
    if metric == 2:
        return -sum(orig[0] if o == "M" else orig[1] if o == "X" else orig[2] for o in ops)
    if metric == 3:
        s, last = 0, ""
        for o in ops:
            s -= orig[0] if o == "M" else orig[1] if o == "X" else orig[3] + (0 if last == o else orig[2])
            last = o
        return s
    s, i = 0, 0
    while i < len(ops):
        j = i
        while j < len(ops) and ops[j] == ops[i]:
            j += 1
        L, o = j - i, ops[i]
        s -= orig[0] * L if o == "M" else orig[1] * L if o == "X" else min(orig[2] + orig[3] * L, orig[4] + orig[5] * L)
        i = j
    return s


def line(metric, orig, score_only, biwfa, r, ops, n, m, corrected=False):
    status = int(r["status"])
    completed = status == 5
    failed_bi = biwfa and score_only and not completed
    no_alignment = failed_bi or (not biwfa and status in (6, 2) and int(r["end_offset"]) == NULL)
    ev, eh, wfa_score = n, m, int(r["score"])
    if not biwfa and status in (6, 2):
        ev, eh = _wrap(int(r["end_offset"]) - int(r["end_k"])), int(r["end_offset"])
        if int(r["end_score"]) >= 0:
            wfa_score = int(r["end_score"])
    if score_only and corrected and no_alignment:
        out = -1
    elif failed_bi:
        out = INT_MIN
    elif not score_only:
        out = -1 if not ops else classic_score(metric, orig, ops)
    elif metric in (0, 1):
        out = wfa_score
    elif orig[0] < 0:
        out = _wrap(_wrap(-orig[0] * _wrap(ev + eh)) - wfa_score)
        out = int(out / 2)
    else:
        out = -wfa_score
    cg = "-" if (score_only or not ops) else rle(ops)
    return f"{out}\t{cg}"
