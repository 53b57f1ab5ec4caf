"""GPU parity: the CUDA path through the C ABI against the oracle.

Integer work, so the bar is bit-exact: score, status, CIGAR (tie-breaks
included), CIGAR score/end and alignment end position of every pair.
"""
import random

import numpy as np
import pytest

import cli_format
import oracle as O
from _pkg import load
from test_emu_vs_oracle import CORR_PENS, HEUR, PENS
from test_oracle_unit import lcg_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return load()


def pack(pairs):
    buf, po, pl, to, tl = bytearray(), [], [], [], []
    for p, t in pairs:
        po.append(len(buf)); buf += p; pl.append(len(p))
        to.append(len(buf)); buf += t; tl.append(len(t))
    buf += b"\0" * 16
    return np.frombuffer(bytes(buf), np.uint8), po, pl, to, tl


def gpu_batch(pkg, metric, pen, pairs, compute=True, span=0, free=None, hk=0, hp=(0, 0, 0),
              extension=False, packed=False, memory="high", compat=0):
    a = pkg.WavefrontAligner(metric, pen)
    a.set_alignment_scope(compute)
    a.set_memory_mode(memory)
    a.set_compat(compat == 1)
    if hk:
        a.set_heuristic(hk, *hp)
    if extension:
        a.set_alignment_extension()
    elif span:
        a.set_alignment_free_ends(*free)
    if packed:
        from wfa_b200 import synth
        ps = synth.PairSet(*pack(pairs))
        words, pwo, two = synth.pack2bits(ps)
        res, cig = a.align_batch(np.concatenate([words, np.zeros(4, np.uint32)]), pwo, ps.p_len,
                                 two, ps.t_len, packed=True, span=int(span or extension))
    else:
        seq, po, pl, to, tl = pack(pairs)
        res, cig = a.align_batch(seq, po, pl, to, tl, span=int(span or extension))
    cigars = [cig[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes().decode()
              for r in res]
    return res, cigars


def oracle_one(metric, pen, p, t, compute, span, free, hk, hp, extension, memory="high", compat=0):
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


def compare(pkg, metric, pen, pairs, compute=True, span=0, free=None, hk=0, hp=(0, 0, 0),
            extension=False, packed=False, memory="high", compat=0):
    res, cig = gpu_batch(pkg, metric, pen, pairs, compute, span, free, hk, hp, extension, packed,
                         memory, compat)
    for i, (p, t) in enumerate(pairs):
        s, st, ops, ep, (cs, ev, eh) = oracle_one(metric, pen, p, t, compute, span, free, hk, hp,
                                                  extension, memory, compat)
        r = res[i]
        got = (int(r["score"]), int(r["status"]), cig[i] if compute else "",
               (int(r["end_score"]), int(r["end_k"]), int(r["end_offset"])))
        assert got == (s, st, ops, ep), (metric, pen, i, got[:2], (s, st))
        if compute:
            assert (int(r["cigar_score"]), int(r["end_v"]), int(r["end_h"])) == (cs, ev, eh), i


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("compute", [True, False])
def test_end2end(pkg, metric, pen, compute):
    pairs = lcg_pairs(211 + metric, 120, 300)
    compare(pkg, metric, pen, pairs, compute=compute)
    compare(pkg, metric, pen, pairs[:60], compute=compute, packed=True)


@pytest.mark.parametrize("metric,pen", PENS)
def test_endsfree_and_extension(pkg, metric, pen):
    r = random.Random(metric)
    for p, t in lcg_pairs(223 + metric, 12, 200):
        free = [r.randrange(0, len(p) // 4 + 1), r.randrange(0, len(p) // 4 + 1),
                r.randrange(0, len(t) // 4 + 1), r.randrange(0, len(t) // 4 + 1)]
        compare(pkg, metric, pen, [(p, t)], span=1, free=free)
    if metric >= 2:
        compare(pkg, metric, pen, lcg_pairs(227 + metric, 60, 200), extension=True)


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("h,hp", [("wfa-adaptive", (10, 50, 1)), ("xdrop", (20, 1, 0)),
                                  ("xdrop", (20, 3, 0)), ("zdrop", (20, 1, 0)),
                                  ("banded-static", (-5, 5, 0)), ("banded-adaptive", (-3, 3, 1))])
def test_heuristics(pkg, metric, pen, h, hp):
    if h in ("xdrop", "zdrop") and metric in (0, 1):
        pytest.skip("drops are rejected with edit/indel")
    compare(pkg, metric, pen, lcg_pairs(233 + metric, 60, 300), hk=HEUR[h], hp=hp)
    if metric >= 2 and h in ("xdrop", "zdrop"):
        compare(pkg, metric, pen, lcg_pairs(239 + metric, 30, 200), hk=HEUR[h], hp=hp,
                extension=True)


def test_edges(pkg):
    edge = [(b"", b""), (b"A", b""), (b"", b"ACGT"), (b"A", b"C"), (b"A", b"A"),
            (b"ACGT" * 40, b"ACGT" * 40), (b"AAAAAAAA", b"CCCCCCCC"),
            (b"ACGTTTTTTTTTTACGT", b"ACGTACGT"), (b"A" * 700, b"C" * 700)]
    for metric, pen in PENS:
        compare(pkg, metric, pen, edge)
        compare(pkg, metric, pen, edge, packed=True)


def test_retry_escalation(pkg):
    """Pairs whose wavefronts outgrow the first scratch configuration are
    re-run with more scratch and still match."""
    r = random.Random(5)
    big = (bytes(r.choice(b"ACGT") for _ in range(3000)), bytes(r.choice(b"ACGT") for _ in range(2900)))
    pairs = lcg_pairs(241, 40, 150) + [big] + lcg_pairs(242, 40, 150)
    compare(pkg, 3, [0, 4, 6, 2], pairs)
    compare(pkg, 1, None, pairs)


@pytest.mark.parametrize("metric,pen", PENS)
@pytest.mark.parametrize("memory", ["med", "low"])
def test_med_low_piggyback(pkg, metric, pen, memory):
    """Med/low memory with an alignment: the piggyback backtrace's CIGARs."""
    compare(pkg, metric, pen, lcg_pairs(261 + metric, 60, 300), memory=memory)
    compare(pkg, metric, pen, lcg_pairs(263 + metric, 30, 200), packed=True, memory=memory)


@pytest.mark.parametrize("metric,pen", PENS)
def test_med_low_piggyback_spans_and_heuristics(pkg, metric, pen):
    r = random.Random(metric + 17)
    for p, t in lcg_pairs(267 + metric, 12, 200):
        free = [r.randrange(0, len(p) // 3 + 1), r.randrange(0, len(p) // 3 + 1),
                r.randrange(0, len(t) // 3 + 1), r.randrange(0, len(t) // 3 + 1)]
        compare(pkg, metric, pen, [(p, t)], span=1, free=free, memory="med")
    if metric >= 2:
        compare(pkg, metric, pen, lcg_pairs(269 + metric, 30, 200), extension=True, memory="low")
        compare(pkg, metric, pen, lcg_pairs(271 + metric, 30, 250), hk=2, hp=(20, 1, 0), memory="med")
    compare(pkg, metric, pen, lcg_pairs(273 + metric, 30, 250), hk=1, hp=(10, 50, 1), memory="med")
    compare(pkg, metric, pen, lcg_pairs(275 + metric, 30, 250), hk=5, hp=(-3, 3, 1), memory="low")


@pytest.mark.parametrize("memory", ["high", "med", "low"])
def test_reference_unit_cases_in_every_memory_mode(pkg, memory):
    """src/aligner.rs:3890-3943: empty sequences give score 0 and an empty
    CIGAR; a begin-free seed at score 0 starts the CIGAR at its position."""
    for metric, pen in [(1, None), (3, [0, 4, 6, 2])]:
        for endsfree in (False, True):
            a = pkg.WavefrontAligner(metric, pen)
            a.set_memory_mode(memory)
            a.set_alignment_scope(True)
            if endsfree:
                a.set_alignment_free_ends(0, 0, 0, 0)
                s = a.align_endsfree(b"", b"")
            else:
                s = a.align_end2end(b"", b"")
            assert s == 0 and a.status() == 5 and a.cigar().operations == b""  # Completed
    a = pkg.WavefrontAligner(2, [0, 3, 3])
    a.set_memory_mode(memory)
    a.set_alignment_scope(True)
    a.set_alignment_free_ends(0, 0, 4, 11)
    a.align_endsfree(b"G", b"TCGGGACATCGAG")
    assert a.cigar().to_string_rle() == "2I1M10I"


@pytest.mark.parametrize("metric,pen", CORR_PENS)
def test_corrected_endsfree(pkg, metric, pen):
    """Compat::Corrected ends-free with a match reward (the end candidate and
    the diagonal pruning), one batch per free-end setting."""
    pairs = lcg_pairs(281 + metric, 40, 200)
    for free in ([0, 40, 0, 40], [200, 200, 200, 200], [10, 60, 0, 200]):
        fr = [[min(f, len(p) if i < 2 else len(t)) for i, f in enumerate(free)] for p, t in pairs]
        for (p, t), f in zip(pairs, fr):
            compare(pkg, metric, pen, [(p, t)], span=1, free=f, compat=1)
    compare(pkg, metric, pen, pairs, extension=True, compat=1)
    compare(pkg, metric, pen, pairs, extension=True, memory="med", compat=1)
    compare(pkg, metric, pen, pairs, compute=False, extension=True, compat=1)


@pytest.mark.parametrize("metric,pen", CORR_PENS)
def test_corrected_dominance_and_heuristics(pkg, metric, pen):
    pairs = lcg_pairs(283 + metric, 40, 200)
    for i, (p, t) in enumerate(pairs[:16]):
        b, e = 1 + i % 5, 0 if i % 2 else 16
        free = [min(b, len(p)), min(e, len(p)), min(b, len(t)), min(e, len(t))]
        compare(pkg, metric, pen, [(p, t)], span=1, free=free, memory=["high", "low"][i % 2], compat=1)
    for hk, hp in ((4, (-20, 20, 0)), (2, (30, 1, 0)), (3, (30, 1, 0)), (1, (10, 50, 1))):
        compare(pkg, metric, pen, pairs, hk=hk, hp=hp, compat=1)
        compare(pkg, metric, pen, pairs, hk=hk, hp=hp, memory="med", compat=1)


def test_corrected_reference_cases(pkg, golden):
    """tests/corrected_endsfree.rs issue_37_repeat_shift (the corrected CIGAR
    and real score) and tests/corrected_zdrop.rs issue_22_corrected_modes_agree."""
    a = pkg.WavefrontAligner(3, [-5, 4, 0, 8])
    a.set_compat(True)
    a.set_alignment_scope(True)
    a.set_alignment_free_ends(12, 12, 11, 11)
    w = a.align_endsfree(b"ACGTACGTACGT", b"ACGACGTACGT")
    assert (5 * 23 - w) // 2 == 47 and a.cigar().operations == b"MMMDMMMMMMMM"
    x = golden["extra"]["issue22_zdrop_high"]
    (p, t), = x["pairs"]
    got = set()
    for memory in ("high", "med", "low"):
        a = pkg.WavefrontAligner(3, x["penalties"])
        a.set_compat(True)
        a.set_memory_mode(memory)
        a.set_alignment_scope(True)
        a.set_heuristic("zdrop", *x["zdrop"])
        a.align_end2end(p.encode(), t.encode())
        got.add(cli_format.classic_score(3, x["penalties"] + [0, 0], a.cigar().operations.decode()))
    assert got == {x["cigar_affine_score"]}


def test_med_low_picks_fixed_at_compute_time(pkg):
    """Med/low where a later step changes what a kernel read: banded-adaptive
    cutoffs emptying I/D of the score M was just computed from (ends-free,
    match reward), and C-mode Z-drop ends read on a dead cell."""
    r = random.Random(4242)
    pairs = []
    for _ in range(40):
        n = r.randint(40, 400)
        p = bytes(r.choice(b"ACGT") for _ in range(n))
        t = bytearray()
        for c in p:
            u = r.random()
            if u < 0.05: t += bytes([r.choice(b"ACGT")])
            elif u < 0.10: t += bytes([r.choice(b"ACGT"), c])
            elif u < 0.15: pass
            else: t.append(c)
        pairs.append((p, bytes(t)))
    for memory in ("med", "low"):
        for p, t in pairs:
            free = [len(p) // 5, len(p) // 5, len(t) // 5, len(t) // 5]
            compare(pkg, 3, [-3, 5, 3, 2], [(p, t)], span=1, free=free, hk=5, hp=(-8, 8, 1), memory=memory)
            compare(pkg, 4, [-1, 4, 6, 2, 24, 1], [(p, t)], span=1, free=free, hk=5, hp=(-8, 8, 1),
                    memory=memory)
        compare(pkg, 4, [-1, 4, 6, 2, 24, 1], pairs, hk=3, hp=(20, 1, 0), memory=memory)
        compare(pkg, 4, [-1, 4, 6, 2, 24, 1], pairs, extension=True, hk=3, hp=(20, 1, 0), memory=memory)


def test_med_low_compaction_and_memory(pkg):
    """Pairs whose alignments pass score 6000 (the reference's compaction
    probe) with max_memory_compact at 64 KiB: the backtrace buffer is
    compacted and every CIGAR still equals the oracle's (which never
    compacts).  Med/low hold no history, so a pair needs less device memory
    than in high memory."""
    r = random.Random(31)
    pairs = []
    for n in (7000, 8000):
        p = bytes(r.choice(b"ACGT") for _ in range(n))
        t = bytearray()
        for c in p:
            u = r.random()
            if u < 0.08: t += bytes([r.choice(b"ACGT")])
            elif u < 0.14: t += bytes([r.choice(b"ACGT"), c])
            elif u < 0.20: pass
            else: t.append(c)
        pairs.append((p, bytes(t)))
    for memory in ("med", "low"):
        a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
        a.set_alignment_scope(True)
        a.set_memory_mode(memory)
        a.set_max_memory_compact(64 << 10)
        seq, po, pl, to, tl = pack(pairs)
        res, cig = a.align_batch(seq, po, pl, to, tl)
        a.close()
        for i, (p, t) in enumerate(pairs):
            o = O.OracleAligner(3, [0, 4, 6, 2])
            o.set_alignment_scope(True)
            o.set_memory_mode(memory)
            s = o.align_end2end(p, t)
            assert s > 6000
            rr = res[i]
            got = cig[rr["cigar_begin"]:rr["cigar_begin"] + rr["cigar_length"]].tobytes()
            assert (int(rr["score"]), int(rr["status"]), got) == (s, o.status(), o.cigar()[0]), (memory, i)
    # Device bytes per pair in flight: C4-shaped pairs (0.5-5 kbp cores with
    # flanks), extension span, CIGAR, med against high memory.
    from wfa_b200 import synth
    ps = synth.config4(64, synth.SEED_BASE + 44)
    sizes = {}
    for memory in ("high", "med"):
        a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
        a.set_alignment_scope(True)
        a.set_memory_mode(memory)
        a.set_alignment_extension()
        a.align_batch(ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len, span=1)
        sizes[memory] = a.last_slice_bytes()
        a.close()
    assert 0 < sizes["med"] < sizes["high"], sizes


def test_med_low_long_pairs(pkg):
    """Pairs long enough to outgrow the first history size re-run and match."""
    r = random.Random(29)
    pairs = []
    for n in (1500, 3000):
        p = bytes(r.choice(b"ACGT") for _ in range(n))
        t = bytearray(p)
        for _ in range(n // 12):
            t[r.randrange(len(t))] = r.choice(b"ACGT")
        pairs.append((p, bytes(t)))
    for metric, pen in [(1, None), (3, [0, 4, 6, 2]), (4, [0, 4, 6, 2, 24, 1])]:
        compare(pkg, metric, pen, pairs + lcg_pairs(277, 20, 200), memory="med")


def test_plain_calls_and_golden_cli(pkg, golden):
    """The plain per-call form reproduces the reference's CLI golden lines."""
    for case in golden["cases"]:
        if case["memory"] not in ("high", "med", "low"):
            continue
        metric = O.METRICS[case["algo"]]
        pen = [int(x) for x in case["penalties"].split(",")] if case["penalties"] else O.DEFAULT_PEN[metric]
        so = case["score_only"]
        a = pkg.WavefrontAligner(metric, pen)
        a.set_alignment_scope(not so)
        a.set_memory_mode(case["memory"])
        a.set_compat(case.get("no_c_compat", False))
        if case["heuristic"]:
            a.set_heuristic(case["heuristic"], *[int(x) for x in case["hparams"].split(",")])
        span_s = case["span"]
        if span_s in ("extension", "extend"):
            a.set_alignment_extension()
        lines = []
        for p, t in case["pairs"]:
            pb, tb = p.encode(), t.encode()
            if span_s == "global":
                s = a.align_end2end(pb, tb)
            else:
                if span_s not in ("extension", "extend"):
                    fr = [float(x) for x in span_s.split(",")[1:]]
                    a.set_alignment_free_ends(O.nominal_prop(len(pb), fr[0]), O.nominal_prop(len(pb), fr[1]),
                                              O.nominal_prop(len(tb), fr[2]), O.nominal_prop(len(tb), fr[3]))
                s = a.align_endsfree(pb, tb)
            c = a.cigar()
            es, ek, eo = a.alignment_end_pos
            rec = {"score": s, "status": a.status(), "end_score": es, "end_k": ek, "end_offset": eo}
            orig = (pen + [0] * 6)[:6]
            lines.append(cli_format.line(metric, orig, so, False, rec, c.operations.decode(), len(pb), len(tb),
                                         case.get("no_c_compat", False)))
        assert lines == case["expected"], case["name"]


def test_config1_full(pkg):
    """10,000 x 100 bp gap-affine pairs (the plain small workload), every pair."""
    from wfa_b200 import synth
    ps = synth.config1()
    a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    res, cig = a.align_batch(ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len)
    secs, scores, status, hashes = O.batch(3, [0, 4, 6, 2], ps.buf.tobytes(), ps.p_off, ps.p_len,
                                           ps.t_off, ps.t_len, threads=8)
    assert np.array_equal(res["score"], scores)
    assert np.array_equal(res["status"], status)
    for i in range(len(ps)):
        r = res[i]
        ops = cig[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes()
        h = 1469598103934665603
        for c in ops:
            h = ((h ^ c) * 1099511628211) & (2**64 - 1)
        assert (h - 2**64 if h >= 2**63 else h) == hashes[i], i


def test_config2_sample_packed(pkg):
    """Short-read batch shape (100-150 bp, 0-4% edits), 2-bit packed input,
    100,000 pairs, every pair against the oracle."""
    from wfa_b200 import synth
    ps = synth.uniform_pairs(100_000, 100, 150, 0.0, 0.04, synth.SEED_BASE + 2)
    words, pwo, two = synth.pack2bits(ps)
    a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    res, cig = a.align_batch(np.concatenate([words, np.zeros(4, np.uint32)]), pwo, ps.p_len, two,
                             ps.t_len, packed=True)
    secs, scores, status, hashes = O.batch(3, [0, 4, 6, 2], ps.buf.tobytes(), ps.p_off, ps.p_len,
                                           ps.t_off, ps.t_len, threads=8)
    assert np.array_equal(res["score"], scores)
    assert np.array_equal(res["status"], status)
    got = O.hash_ops(cig, res["cigar_begin"].astype(np.int64), res["cigar_length"], 8)
    assert np.array_equal(got, hashes)


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
@pytest.mark.parametrize("metric,pen", PENS)
def test_lane_group_widths(pkg, metric, pen, lanes):
    """Every lane-group width of the end-to-end kernel, every metric, both
    encodings, score-only and CIGAR: 100-400 bp pairs at 0-15 % edits (some
    wavefronts wider than the shared-memory ring slots, which spill), every
    pair against the oracle."""
    from wfa_b200 import synth
    ps = synth.uniform_pairs(3000, 100, 400, 0.0, 0.15, 0x5EED0000 + 300 + metric)
    words, pwo, two = synth.pack2bits(ps)
    words = np.concatenate([words, np.zeros(4, np.uint32)])
    for compute in (True, False):
        _, scores, status, hashes = O.batch(metric, pen, ps.buf.tobytes(), ps.p_off, ps.p_len,
                                            ps.t_off, ps.t_len, compute_alignment=compute, threads=8)
        for packed in (True, False):
            a = pkg.WavefrontAligner(metric, pen)
            a.set_alignment_scope(compute)
            a.set_lanes_per_pair(lanes)
            if packed:
                res, cig = a.align_batch(words, pwo, ps.p_len, two, ps.t_len, packed=True)
            else:
                res, cig = a.align_batch(ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len)
            # (rings too large for a block of narrow groups run wider groups)
            assert a.last_lanes_per_pair() >= lanes
            a.close()
            assert np.array_equal(res["score"], scores), (compute, packed)
            assert np.array_equal(res["status"], status), (compute, packed)
            if compute:
                got = O.hash_ops(cig, res["cigar_begin"].astype(np.int64), res["cigar_length"], 8)
                assert np.array_equal(got, hashes), packed


def test_device_api_matches_host_api(pkg):
    import torch
    from wfa_b200 import synth
    ps = synth.uniform_pairs(5000, 100, 150, 0.0, 0.04, 77)
    words, pwo, two = synth.pack2bits(ps)
    a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    res_h, cig_h = a.align_batch(np.concatenate([words, np.zeros(4, np.uint32)]), pwo, ps.p_len,
                                 two, ps.t_len, packed=True)
    dev = torch.device("cuda:0")
    w = torch.from_numpy(np.concatenate([words, np.zeros(4, np.uint32)]).view(np.int32)).to(dev)
    t_po = torch.from_numpy(pwo).to(dev)
    t_pl = torch.from_numpy(ps.p_len).to(dev)
    t_to = torch.from_numpy(two).to(dev)
    t_tl = torch.from_numpy(ps.t_len).to(dev)
    caps = 2 * (ps.p_len.astype(np.int64) + ps.t_len) + 1
    coff = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    t_co = torch.from_numpy(coff).to(dev)
    cig = torch.zeros(int(caps.sum()) + 16, dtype=torch.uint8, device=dev)
    res = torch.zeros(len(ps) * 10, dtype=torch.int32, device=dev)
    a.align_batch_device(w.data_ptr(), w.numel() * 4, t_po.data_ptr(), t_pl.data_ptr(),
                         t_to.data_ptr(), t_tl.data_ptr(), len(ps), res.data_ptr(), cig.data_ptr(),
                         t_co.data_ptr(), int(caps.sum()), packed=True)
    torch.cuda.synchronize()
    rd = res.cpu().numpy().view(res_h.dtype)
    cd = cig.cpu().numpy()
    assert np.array_equal(rd["score"], res_h["score"])
    assert np.array_equal(rd["status"], res_h["status"])
    for i in range(0, len(ps), 97):
        a_ops = cd[coff[i] + rd["cigar_begin"][i]: coff[i] + rd["cigar_begin"][i] + rd["cigar_length"][i]]
        b_ops = cig_h[res_h["cigar_begin"][i]: res_h["cigar_begin"][i] + res_h["cigar_length"][i]]
        assert a_ops.tobytes() == b_ops.tobytes(), i


def test_host_batch_across_chunks(pkg):
    """A host-buffer batch large enough to run in several chunks (short first
    and last ones), with empty patterns and one long pair, matches the
    device-buffer call pair by pair, and its packed CIGARs tile the output."""
    import torch
    from wfa_b200 import synth
    base = synth.uniform_pairs(200000, 100, 150, 0.0, 0.04, 91)
    r = random.Random(3)
    lp = bytes(r.choice(b"ACGT") for _ in range(3000))
    lt = bytearray(lp)
    for _ in range(250):
        lt[r.randrange(len(lt))] = r.choice(b"ACGT")
    buf = np.concatenate([base.buf, np.frombuffer(lp + bytes(lt), np.uint8)])
    p_off, p_len = base.p_off.copy(), base.p_len.copy()
    t_off, t_len = base.t_off.copy(), base.t_len.copy()
    p_len[::997] = 0
    p_off[100000], p_len[100000] = len(base.buf), len(lp)
    t_off[100000], t_len[100000] = len(base.buf) + len(lp), len(lt)
    ps = synth.PairSet(buf, p_off, p_len, t_off, t_len)
    words, pwo, two = synth.pack2bits(ps)
    words = np.concatenate([words, np.zeros(4, np.uint32)])
    a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    res_h, cig_h = a.align_batch(words, pwo, ps.p_len, two, ps.t_len, packed=True)
    dev = torch.device("cuda:0")
    w = torch.from_numpy(words.view(np.int32)).to(dev)
    caps = 2 * (ps.p_len.astype(np.int64) + ps.t_len) + 1
    coff = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    args = [torch.from_numpy(x).to(dev) for x in (pwo, ps.p_len, two, ps.t_len, coff)]
    cig = torch.zeros(int(caps.sum()) + 16, dtype=torch.uint8, device=dev)
    res = torch.zeros(len(ps) * 10, dtype=torch.int32, device=dev)
    a.align_batch_device(w.data_ptr(), w.numel() * 4, args[0].data_ptr(), args[1].data_ptr(),
                         args[2].data_ptr(), args[3].data_ptr(), len(ps), res.data_ptr(), cig.data_ptr(),
                         args[4].data_ptr(), int(caps.sum()), packed=True)
    torch.cuda.synchronize()
    rd = res.cpu().numpy().view(res_h.dtype)
    cd = cig.cpu().numpy()
    for f in ("score", "status", "cigar_length", "cigar_score", "end_v", "end_h"):
        assert np.array_equal(rd[f], res_h[f]), f
    assert res_h["cigar_length"][100000] >= 3000
    # The packed CIGARs tile the output without gaps or overlaps.
    beg = res_h["cigar_begin"].astype(np.int64)
    order = np.argsort(beg, kind="stable")
    ends = beg[order] + res_h["cigar_length"][order]
    assert beg[order][0] == 0 and np.array_equal(beg[order][1:], ends[:-1])
    for i in list(range(0, len(ps), 1013)) + [100000, len(ps) - 1]:
        a_ops = cd[coff[i] + rd["cigar_begin"][i]: coff[i] + rd["cigar_begin"][i] + rd["cigar_length"][i]]
        b_ops = cig_h[res_h["cigar_begin"][i]: res_h["cigar_begin"][i] + res_h["cigar_length"][i]]
        assert a_ops.tobytes() == b_ops.tobytes(), i


def test_async_batches_match_the_blocking_call(pkg):
    """wfa_batch_submit / poll / wait: three batches queued at once give the
    results of wfa_batch_align, in order."""
    from wfa_b200 import synth
    a = pkg.WavefrontAligner(3, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    sets = [synth.uniform_pairs(3000, 100, 150, 0.0, 0.04, 500 + i) for i in range(3)]
    tickets = [a.submit_batch(ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len) for ps in sets]
    import time
    t0 = time.time()
    while not a.poll_batch(tickets[0]):
        assert time.time() - t0 < 120
        time.sleep(0.001)
    got = [a.wait_batch(t) for t in tickets]
    for ps, (res, cig) in zip(sets, got):
        ref_res, ref_cig = a.align_batch(ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len)
        assert np.array_equal(res, ref_res)
        assert cig[:int(res["cigar_length"].sum())].tobytes() == ref_cig[:int(ref_res["cigar_length"].sum())].tobytes()
    a.close()
