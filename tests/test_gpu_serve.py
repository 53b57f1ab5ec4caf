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


def test_same_alone_and_in_mix(pkg):
    reqs = mix(41)
    # (n + m)^2 / 4 above 4 MiB, i.e. n + m above 4096, runs in BiWFA; the
    # short lane takes n + m up to 1024.
    srv = pkg.Server(pkg.GAP_AFFINE, PEN, workers=2, short_workers=2, biwfa_workers=1,
                     max_batch_pairs=16, biwfa_above_bytes=4 << 20)
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
