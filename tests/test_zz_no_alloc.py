"""The no-allocation device batch (wfa_batch_align_device_noalloc) against the
ordinary device batch (wfa_batch_align_device), through the C ABI.

The no-allocation form exists for callers that must not allocate device
memory themselves: a plug-in whose host program's allocator already holds the
device memory, or code that cannot afford the device-wide wait of a cudaFree.
Its scratch is one fixed device array shared by every call on a device, so
these tests also check that a second call in a row, which finds the array as
the first call left it, still gives the same results.  All values are
integers: the comparison is exact.

This file is named to be collected last, after every other test.
"""
import os
import sys

import numpy as np
import pytest

from _pkg import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return load()


def _device_batch(ps, packed):
    """Device copies of a PairSet (2-bit packed or ASCII) and output slots."""
    import torch
    from wfa_b200 import synth
    dev = torch.device("cuda:0")
    if packed:
        words, po, to = synth.pack2bits(ps)
        seq = np.concatenate([words, np.zeros(4, np.uint32)]).view(np.uint8)
    else:
        seq = np.concatenate([ps.buf, np.zeros(16, np.uint8)])
        po, to = ps.p_off, ps.t_off
    caps = 2 * (ps.p_len.astype(np.int64) + ps.t_len) + 1
    coff = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    return {"seq": t(seq), "po": t(po), "pl": t(ps.p_len), "to": t(to), "tl": t(ps.t_len),
            "co": t(coff), "coff": coff, "cap": int(caps.sum()), "n": len(ps), "packed": packed}


def _outputs(d):
    import torch
    dev = torch.device("cuda:0")
    res = torch.full((d["n"] * 10,), -7, dtype=torch.int32, device=dev)
    cig = torch.full((d["cap"] + 16,), 0xAB, dtype=torch.uint8, device=dev)
    return res, cig


def _run(a, d, noalloc, span=0, out=None):
    """One call of either entry point into fresh (poisoned) output buffers,
    or into `out` (results, CIGAR slots) when given."""
    import torch
    res, cig = out if out is not None else _outputs(d)
    fn = a.align_batch_device_noalloc if noalloc else a.align_batch_device
    fn(d["seq"].data_ptr(), d["seq"].numel(), d["po"].data_ptr(), d["pl"].data_ptr(),
       d["to"].data_ptr(), d["tl"].data_ptr(), d["n"], res.data_ptr(), cig.data_ptr(),
       d["co"].data_ptr(), d["cap"], packed=d["packed"], span=span)
    torch.cuda.synchronize()
    return res.cpu().numpy(), cig.cpu().numpy()


def _same(a, d, span=0, compute=True):
    ref_res, ref_cig = _run(a, d, noalloc=False, span=span)
    got_res, got_cig = _run(a, d, noalloc=True, span=span)
    assert np.array_equal(got_res, ref_res)
    if compute:
        r = got_res.reshape(-1, 10)
        for i in range(d["n"]):
            b = d["coff"][i] + r[i, 2]
            assert got_cig[b:b + r[i, 3]].tobytes() == ref_cig[b:b + r[i, 3]].tobytes(), i
    return got_res


def test_two_calls_in_a_row_match_the_device_batch(pkg):
    from wfa_b200 import synth
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    # Call 1: short reads, 2-bit packed.
    short = _device_batch(synth.uniform_pairs(20_000, 100, 150, 0.0, 0.04, 901), packed=True)
    res1 = _same(a, short)
    assert np.all(res1.reshape(-1, 10)[:, 1] == 5)  # every pair END_REACHED
    # Call 2, right after: longer, noisier pairs in ASCII, whose M histories
    # outgrow the first round's slices (re-run with larger ones).
    long_ = _device_batch(synth.uniform_pairs(3_000, 300, 1500, 0.08, 0.12, 902), packed=False)
    res2 = _same(a, long_)
    assert np.all(res2.reshape(-1, 10)[:, 1] == 5)
    a.close()


def test_matches_the_oracle(pkg):
    """Scores, statuses and CIGARs of a no-allocation call equal the oracle's
    (the CPU restatement of the reference) pair for pair."""
    from wfa_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ps = synth.uniform_pairs(5_000, 100, 400, 0.0, 0.08, 906)
    d = _device_batch(ps, packed=True)
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    res, cig = _run(a, d, noalloc=True)
    a.close()
    r = res.view(pkg.RESULT_DTYPE)
    _, sc, st, hs = O.batch(3, [0, 4, 6, 2], ps.buf.tobytes(), ps.p_off, ps.p_len, ps.t_off,
                            ps.t_len, threads=os.cpu_count() or 1)
    gh = O.hash_ops(cig, d["coff"] + r["cigar_begin"], r["cigar_length"])
    assert np.array_equal(r["score"], sc)
    assert np.array_equal(r["status"], st)
    assert np.array_equal(gh, hs)


def test_allocates_no_device_memory(pkg):
    """Free device memory is the same before and after a call that re-runs
    pairs with larger slices (the path that would grow an ordinary scratch).
    The handle, the inputs and the outputs are made first; one call before
    the measured one loads the module that holds the array."""
    import torch
    from wfa_b200 import synth
    ps = synth.uniform_pairs(4_000, 300, 1500, 0.08, 0.12, 907)
    d = _device_batch(ps, packed=True)
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    out = _outputs(d)
    _run(a, d, noalloc=True, out=out)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _run(a, d, noalloc=True, out=out)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert a.last_rerun_pairs() > 0  # the measured call did re-run pairs
    assert free1 == free0
    a.close()


def test_more_reruns_than_one_round_holds(pkg):
    """More pairs to re-run than one round gathers (65,536): the rest are
    gathered in later rounds.  Score-only and ends-free calls as well."""
    from wfa_b200 import synth
    ps = synth.uniform_pairs(70_000, 400, 500, 0.10, 0.12, 903)
    d = _device_batch(ps, packed=True)
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    _same(a, d)
    # The call just made (the no-allocation one) re-ran more pairs than one
    # gathering round holds, so the later rounds were exercised.
    assert a.last_rerun_pairs() > 65_536
    a.set_alignment_scope(False)
    _same(a, d, compute=False)
    e = pkg.WavefrontAligner(pkg.EDIT, None)
    e.set_alignment_scope(True)
    e.set_alignment_free_ends(20, 20, 20, 20)
    _same(e, d, span=1)
    a.close()
    e.close()


def test_limits_are_reported(pkg):
    from wfa_b200 import synth
    a = pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    a.set_alignment_scope(True)
    too_long = _device_batch(synth.uniform_pairs(4, 2100, 2100, 0.01, 0.01, 904), packed=True)
    with pytest.raises(RuntimeError, match="WFA_NOALLOC_MAX_LEN_SUM"):
        _run(a, too_long, noalloc=True)
    short = _device_batch(synth.uniform_pairs(8, 100, 100, 0.01, 0.01, 905), packed=True)
    with pytest.raises(NotImplementedError):
        _run(a, short, noalloc=True, span=2)
    # The handle still works after the refusals.
    _same(a, short)
    a.close()
