"""The serving loop (continuous batching) on the GPU through the C ABI: every
request gets the same result in a concurrent mix as alone, and that result
is the plain aligner call's in the request's mode (high-memory end-to-end,
or BiWFA above the memory threshold).  Integer results: exact."""
import threading
import time

import numpy as np
import pytest

from _pkg import load

pytestmark = pytest.mark.gpu

PEN = [0, 4, 6, 2]


@pytest.fixture(scope="module")
def pkg():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return load()


def mix(seed):
    from wfa_b200 import synth
    out = []
    for num, lo, hi, rate in [(60, 150, 150, 0.02), (10, 1000, 4000, 0.08), (4, 2500, 3500, 0.10)]:
        ps = synth.uniform_pairs(num, lo, hi, rate, rate, seed + lo)
        out += [ps.pair(i) for i in range(num)]
    r = np.random.default_rng(seed)
    return [out[i] for i in r.permutation(len(out))]


def collect(srv, ids, timeout_s=300):
    got = {}
    t0 = time.time()
    while len(got) < len(ids):
        assert time.time() - t0 < timeout_s, "server did not finish"
        for rec in srv.poll(timeout_ms=200):
            got[rec["id"]] = rec
    return got


def key(rec):
    return (rec["score"], rec["status"], rec["cigar"], rec["cigar_score"], rec["end_v"], rec["end_h"],
            rec["mode"])


@pytest.mark.parametrize("resident", [False, True])
def test_same_alone_and_in_mix(pkg, resident):
    """With resident=True the short lane is a resident stream (a persistent
    kernel taking requests as they come)."""
    reqs = mix(41)
    # (n + m)^2 / 4 above 4 MiB, i.e. n + m above 4096, runs in BiWFA; the
    # short lane takes n + m up to 1024.
    srv = pkg.Server(pkg.GAP_AFFINE, PEN, workers=2, short_workers=2, biwfa_workers=1,
                     max_batch_pairs=16, biwfa_above_bytes=4 << 20, resident=resident)
    try:
        # In the mix: two submitting threads at once.
        ids = [None] * len(reqs)

        def submit(part):
            for i in part:
                ids[i] = srv.submit(*reqs[i])

        th = [threading.Thread(target=submit, args=(range(k, len(reqs), 2),)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        in_mix = collect(srv, ids)
        # Alone: one request at a time through the same server.
        alone = {}
        for i, (p, t) in enumerate(reqs):
            rid = srv.submit(p, t)
            alone[i] = collect(srv, [rid])[rid]
        assert srv.pending() == 0
        failed = [i for i in alone if alone[i]["status"] < 0] + [i for i in ids if in_mix[i]["status"] < 0]
        assert not failed, (failed[:10], srv.last_error())
    finally:
        srv.stop()
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, PEN)
    a.set_alignment_scope(True)
    modes = set()
    for i, (p, t) in enumerate(reqs):
        m = in_mix[ids[i]]
        assert key(m) == key(alone[i]), i
        biwfa = (len(p) + len(t)) ** 2 // 4 > (4 << 20)
        assert m["mode"] == int(biwfa)
        modes.add(m["mode"])
        s = a.align_biwfa(p, t) if biwfa else a.align_end2end(p, t)
        c = a.cigar()
        assert (m["score"], m["status"], m["cigar"]) == (s, a.status(), bytes(c.operations)), i
    assert modes == {0, 1}
    a.close()


def test_biwfa_lane_50kbp_against_the_oracle(pkg):
    """The BiWFA lane with 50 kbp requests beside short ones: every result is
    the oracle's align_biwfa / align_end2end (score, status, CIGAR)."""
    import oracle as O
    from wfa_b200 import synth
    big = synth.pairs_with_lengths([50000], [0.1], 91)
    small = synth.uniform_pairs(6, 120, 150, 0.03, 0.03, 92)
    reqs = [big.pair(0)] + [small.pair(i) for i in range(6)]
    srv = pkg.Server(pkg.GAP_AFFINE, PEN, workers=1, short_workers=1, biwfa_workers=1,
                     biwfa_above_bytes=256 << 20, resident=True)
    try:
        ids = [srv.submit(p, t) for p, t in reqs]
        got = collect(srv, ids, timeout_s=600)
    finally:
        srv.stop()
    for i, (p, t) in enumerate(reqs):
        r = got[ids[i]]
        o = O.OracleAligner(3, PEN)
        o.set_alignment_scope(True)
        biwfa = (len(p) + len(t)) ** 2 // 4 > (256 << 20)
        s = o.align_biwfa(p, t) if biwfa else o.align_end2end(p, t)
        assert biwfa == (i == 0) and r["mode"] == int(biwfa), i
        assert (r["score"], r["status"], r["cigar"]) == (s, o.status(), o.cigar()[0]), (i, len(p))


def _c2_pairs(num, seed):
    from wfa_b200 import synth
    return synth.uniform_pairs(num, 100, 150, 0.0, 0.04, seed)


def _stream_collect(st, want, timeout_s=120):
    got = {}
    t0 = time.time()
    while len(got) < want:
        assert time.time() - t0 < timeout_s, "stream did not finish"
        for r in st.poll(timeout_ms=100):
            got[r["id"]] = r
    return got


def test_stream_matches_the_batch_path(pkg):
    """C2-shaped requests through a resident stream, one at a time and many
    per call, against the batch path (score, status, CIGAR) and the oracle on
    a sample."""
    import oracle as O
    ps = _c2_pairs(3000, 501)
    seq, po, pl, to, tl = ps.buf, ps.p_off, ps.p_len, ps.t_off, ps.t_len
    st = pkg.Stream(pkg.GAP_AFFINE, PEN, max_len_sum=512, capacity=4096)
    try:
        ids = [st.submit(*ps.pair(i)) for i in range(500)]
        first = st.submit_many(seq, po[500:], pl[500:], to[500:], tl[500:])
        assert first == 500 and ids == list(range(500))
        got = _stream_collect(st, len(ps))
        stats = st.stats()
        assert st.pending() == 0
    finally:
        st.stop()
    assert stats["launches"] >= 1 and stats["gave_up"] == 0, stats
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, PEN)
    a.set_alignment_scope(True)
    res, cig = a.align_batch(seq, po, pl, to, tl)
    a.close()
    for i in range(len(ps)):
        r, b = got[i], res[i]
        ops = cig[b["cigar_begin"]:b["cigar_begin"] + b["cigar_length"]].tobytes()
        assert (r["score"], r["status"], r["cigar"]) == (int(b["score"]), int(b["status"]), ops), i
    for i in range(0, len(ps), 97):
        o = O.OracleAligner(3, PEN)
        o.set_alignment_scope(True)
        p, t = ps.pair(i)
        assert got[i]["score"] == o.align_end2end(p, t) and got[i]["cigar"] == o.cigar()[0], i


def test_stream_idle_exit_and_relaunch(pkg):
    """The kernel ends on its own after about a second without requests (its
    polls are bounded) and the next submit launches it again; a full ring
    refuses a submit until poll frees a slot."""
    ps = _c2_pairs(80, 502)
    st = pkg.Stream(pkg.GAP_AFFINE, PEN, max_len_sum=512, capacity=64, blocks_per_sm=1)
    try:
        for i in range(64):
            assert st.submit(*ps.pair(i)) == i
        assert st.submit(*ps.pair(64)) == -7  # WFA_ERR_BUSY
        got = _stream_collect(st, 64)
        time.sleep(3.0)
        st.poll(timeout_ms=50)  # notices the launch that ended
        s1 = st.stats()
        assert s1["idle_exits"] >= 1 and s1["launches"] >= 1, s1
        for i in range(64, 80):
            assert st.submit(*ps.pair(i)) == i
        got.update(_stream_collect(st, 16))
        s2 = st.stats()
        assert s2["launches"] == s1["launches"] + 1 and s2["gave_up"] == 0, (s1, s2)
    finally:
        st.stop()
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, PEN)
    a.set_alignment_scope(True)
    for i in range(80):
        s = a.align_end2end(*ps.pair(i))
        assert (got[i]["score"], got[i]["cigar"]) == (s, bytes(a.cigar().operations)), i
    a.close()
