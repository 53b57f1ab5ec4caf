"""align_benchmark-compatible driver over the GPU library.

The reference's command-line driver (src/bin/align_benchmark.rs) with its
options and output, aligning on the GPU: reads a `.seq` file (alternating
`>pattern` / `<text` lines, prefixes optional, an unpaired last line
ignored), writes one `score<TAB>CIGAR` line per pair in input order, and
prints `Time.Alignment` to stderr.  Global and extension spans, and BiWFA
(`--wfa-memory ultralow`), align the whole file as one batch; the ends-free
span (free ends proportional to each pair's lengths) aligns pair by pair.
The same option checks end the run with status 1 and a message on stderr.

    python wfa2lib-rs_b200/align_benchmark.py -i pairs.seq -o out.alg -a gap-affine-wfa \\
        -g 0,4,6,2 --wfa-memory high
"""
import argparse
import os
import sys
import time

import numpy as np

if __package__:  # imported as part of the package
    from . import aligner as A
    from . import cli_format
else:  # run as a script
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import aligner as A  # noqa: E402
    import cli_format  # noqa: E402

ALGORITHMS = {"indel-wfa": A.INDEL, "edit-wfa": A.EDIT, "gap-linear-wfa": A.GAP_LINEAR,
              "gap-affine-wfa": A.GAP_AFFINE, "gap-affine2p-wfa": A.GAP_AFFINE_2P}
# The driver's default penalties (src/bin/align_benchmark.rs:148-220).
DEFAULT_PENALTIES = {A.INDEL: [], A.EDIT: [], A.GAP_LINEAR: [0, 4, 2], A.GAP_AFFINE: [0, 4, 6, 2],
                     A.GAP_AFFINE_2P: [0, 4, 6, 2, 24, 1]}


def die(msg):
    sys.stderr.write(msg + "\n")
    sys.exit(1)


def nominal_prop(base, factor):
    """src/bin/align_benchmark.rs:257-263: a fraction of the length, or an
    absolute count when above 1."""
    if 0.0 <= factor <= 1.0:
        return int(base * factor) & 0xFFFFFFFF
    return int(factor) & 0xFFFFFFFF


def parse_span(arg):
    """('global'|'extension', None) or ('ends-free', [p0, pf, t0, tf])
    (src/bin/align_benchmark.rs:224-253)."""
    if arg is None or arg == "global":
        return "global", None
    if arg in ("extension", "extend"):
        return "extension", None
    if arg.startswith("ends-free") or arg.startswith("endsfree"):
        try:
            v = [float(x.strip()) for x in arg.split(",")[1:]]
        except ValueError:
            die("Invalid --wfa-span")
        if len(v) != 4:
            die("Invalid --wfa-span")
        return "ends-free", v
    die("Option '--wfa-span' must be in {'global','extension','ends-free'}")


def parse_heuristic(name, params):
    """(name, parameters) as the driver accepts them (:265-306)."""
    try:
        p = [int(x.strip()) for x in params.split(",")] if params else []
    except ValueError:
        die("Invalid heuristic parameter")
    need = {"none": 0, "wfa-adaptive": 3, "xdrop": 2, "zdrop": 2, "banded-static": 2,
            "banded-adaptive": 3}
    if name not in need:
        die(f"Unknown heuristic: {name}")
    if len(p) < need[name]:
        die("Invalid --wfa-heuristic-parameters")
    return name, p[:need[name]]


def read_pairs(path):
    try:
        with open(path, "rb") as f:
            lines = f.read().split(b"\n")
    except OSError as e:
        die(f"Error reading input file {path!r}: {e}")
    if lines and lines[-1] == b"":
        lines.pop()
    lines = [ln[:-1] if ln.endswith(b"\r") else ln for ln in lines]
    pairs = []
    for i in range(0, len(lines) - 1, 2):
        p, t = lines[i], lines[i + 1]
        pairs.append((p[1:] if p.startswith(b">") else p, t[1:] if t.startswith(b"<") else t))
    return pairs


def penalties_for(metric, args):
    src = {A.GAP_LINEAR: args.linear_penalties, A.GAP_AFFINE: args.affine_penalties,
           A.GAP_AFFINE_2P: args.affine2p_penalties}.get(metric)
    if not src:
        return DEFAULT_PENALTIES[metric]
    try:
        return [int(x) for x in src.split(",")]
    except ValueError:
        die("Invalid penalties")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="align_benchmark", add_help=True)
    ap.add_argument("-i", "--input", required=True)
    ap.add_argument("-o", "--output")
    ap.add_argument("-a", "--algorithm", default="gap-affine-wfa")
    ap.add_argument("--wfa-score-only", action="store_true")
    ap.add_argument("--wfa-span")
    ap.add_argument("--wfa-memory")
    ap.add_argument("-p", "--linear-penalties")
    ap.add_argument("-g", "--affine-penalties")
    ap.add_argument("--affine2p-penalties")
    ap.add_argument("--wfa-heuristic")
    ap.add_argument("--wfa-heuristic-parameters")
    ap.add_argument("--wfa-max-steps", type=int)
    ap.add_argument("--no-c-compat", action="store_true",
                    help="fix known C WFA2-lib bugs instead of reproducing them (Compat::Corrected)")
    ap.add_argument("--device", type=int, default=0, help="CUDA device")
    args = ap.parse_args(argv)

    if args.algorithm not in ALGORITHMS:
        die(f"Unknown algorithm: {args.algorithm}")
    metric = ALGORITHMS[args.algorithm]
    pen = penalties_for(metric, args)
    memory = args.wfa_memory or "high"
    if memory not in ("high", "med", "low", "ultralow"):
        die("Option '--wfa-memory' must be in {'high','med','low','ultralow'}")
    biwfa = memory == "ultralow"
    score_only = args.wfa_score_only
    span, fracs = parse_span(args.wfa_span)
    # The reference's preset checks, in its order: BiWFA spans, then drops.
    if biwfa and span != "global":
        die("[WFA] BiWFA ends-free and extension are not supported")
    heur = parse_heuristic(args.wfa_heuristic, args.wfa_heuristic_parameters) if args.wfa_heuristic else None
    drop = heur is not None and heur[0] in ("xdrop", "zdrop")
    if biwfa and drop:
        die("[WFA] BiWFA is not compatible with X-drop/Z-drop heuristics")
    if drop and metric in (A.INDEL, A.EDIT):
        die("[WFA] Heuristics drops are not compatible with 'edit'/'indel' distance metrics")

    try:
        a = A.WavefrontAligner(metric, pen, device=args.device)
    except ValueError as e:
        die(f"[WFA] {e}")
    a.set_alignment_scope(not score_only)
    if args.no_c_compat:
        a.set_compat(True)
    if heur is not None and heur[0] != "none":
        a.set_heuristic(heur[0], *heur[1])
    if not biwfa:
        a.set_memory_mode(memory)
    if args.wfa_max_steps is not None:
        a.set_max_alignment_steps(args.wfa_max_steps)
    if span == "extension":
        a.set_alignment_extension()

    pairs = read_pairs(args.input)
    out = open(args.output, "w") if args.output else sys.stdout
    orig = (list(pen) + [0] * 6)[:6]
    lines = []
    t0 = time.perf_counter()
    try:
        if span == "ends-free":
            for p, t in pairs:
                ends = [nominal_prop(len(p), fracs[0]), nominal_prop(len(p), fracs[1]),
                        nominal_prop(len(t), fracs[2]), nominal_prop(len(t), fracs[3])]
                if ends[0] > len(p) or ends[1] > len(p) or ends[2] > len(t) or ends[3] > len(t):
                    out.write("".join(x + "\n" for x in lines))
                    out.flush()
                    die("[WFA] Ends-free parameters must be not larger than the sequences "
                        f"(P0={ends[0]},Pf={ends[1]},T0={ends[2]},Tf={ends[3]}). Must be "
                        f"(P0<=|P|,Pf<=|P|,T0<=|T|,Tf<=|T|) where (|P|,|T|)=({len(p)},{len(t)})")
                a.set_alignment_free_ends(*ends)
                s = a.align_endsfree(p, t)
                es, ek, eo = a.alignment_end_pos
                rec = {"score": s, "status": a.status(), "end_score": es, "end_k": ek, "end_offset": eo}
                ops = "" if score_only else a.cigar().operations.decode()
                lines.append(cli_format.line(metric, orig, score_only, False, rec, ops, len(p), len(t),
                                             args.no_c_compat))
        elif pairs:
            buf, po, pl, to, tl = bytearray(), [], [], [], []
            for p, t in pairs:
                po.append(len(buf)); buf += p; pl.append(len(p))
                to.append(len(buf)); buf += t; tl.append(len(t))
            buf += b"\0" * 16
            seq = np.frombuffer(bytes(buf), np.uint8)
            res, cig = a.align_batch(seq, po, pl, to, tl,
                                     span=2 if biwfa else (1 if span == "extension" else 0))
            for i, (p, t) in enumerate(pairs):
                r = res[i]
                ops = "" if score_only else \
                    cig[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes().decode()
                lines.append(cli_format.line(metric, orig, score_only, biwfa, r, ops, len(p), len(t),
                                             args.no_c_compat))
    except NotImplementedError as e:
        die(f"[WFA] not available on the GPU build: {e}")
    ms = (time.perf_counter() - t0) * 1000.0
    out.write("".join(x + "\n" for x in lines))
    out.flush()
    n = max(len(pairs), 1)
    sys.stderr.write(f"Time.Alignment {ms:.2f} ms ({len(pairs)} calls, {ms * 1000.0 / n:.2f} us/call)\n")
    a.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
