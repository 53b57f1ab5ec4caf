"""Multi-GPU sharding logic on CPU: the LPT partition and the gather of
per-rank results, with world_size 2 over gloo.  One test stands the
alignment in by a deterministic function of the pair; another aligns real
pairs (with CIGARs) through the CPU build of the device aligner on each rank
and checks rank 0's gathered output against one unsharded oracle run."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from _pkg import load

DT = np.dtype([("score", np.int32), ("status", np.int32)])


def _shard():
    import importlib
    load()
    return importlib.import_module("wfa_b200.shard")


def fake_align(p_len, t_len):
    def fn(idx):
        out = np.empty(len(idx), DT)
        out["score"] = p_len[idx] * 3 - t_len[idx]
        out["status"] = idx % 7
        return out
    return fn


def lengths(n, seed):
    r = np.random.default_rng(seed)
    return r.integers(50, 5000, n).astype(np.int32), r.integers(50, 5000, n).astype(np.int32)


def test_lpt_partition_covers_and_balances():
    sh = _shard()
    p, t = lengths(1000, 1)
    cost = sh.expected_cost(p, t)
    for world in (1, 2, 3, 8):
        parts = sh.lpt_partition(cost, world)
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(len(p)))
        loads = [int(cost[q].sum()) for q in parts]
        # LPT: no rank exceeds the mean by more than the largest single cost
        assert max(loads) - sum(loads) / world <= cost.max()
        assert all(np.array_equal(a, b) for a, b in zip(parts, sh.lpt_partition(cost, world)))


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = _shard()
        p, t = lengths(n, 2)
        out = sh.run_sharded(fake_align(p, t), p, t, rank, world)
        if rank == 0:
            q.put(out.tobytes())
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world", [2])
def test_gather_in_input_order_world2(world):
    n = 301
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = q.get(timeout=120)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    p, t = lengths(n, 2)
    ref = fake_align(p, t)(np.arange(n))
    assert np.frombuffer(got, DT).tobytes() == ref.tobytes()


def _emu_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = _shard()
        import emu_lib
        pairs = _real_pairs()
        p_len = np.array([len(p) for p, _ in pairs], np.int32)
        t_len = np.array([len(t) for _, t in pairs], np.int32)

        def align(idx):
            res, cigars = emu_lib.run(3, [0, 4, 6, 2], [pairs[i] for i in idx], packed=True)
            ops = np.frombuffer("".join(cigars).encode(), np.uint8).copy()
            lens = np.array([len(c) for c in cigars], np.int64)
            res["cigar_begin"] = np.concatenate([[0], np.cumsum(lens)[:-1]])
            res["cigar_length"] = lens
            return res, ops

        out = sh.run_sharded(align, p_len, t_len, rank, world)
        if rank == 0:
            rec, ops = out
            q.put((rec.tobytes(), ops.tobytes()))
    finally:
        dist.destroy_process_group()


def _real_pairs():
    from wfa_b200 import synth
    ps = synth.uniform_pairs(120, 50, 400, 0.0, 0.1, 0x5EED0000 + 77)
    return [ps.pair(i) for i in range(len(ps))]


def test_real_alignments_gathered_with_cigars_world2():
    """Each rank aligns its LPT shard (CIGAR mode, 2-bit packed) with the CPU
    build of the device aligner; rank 0 gets every score, status and CIGAR
    in input order, equal to one unsharded oracle run."""
    import sys
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_emu_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    rec_b, ops_b = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    load()
    import emu_lib
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O
    rec = np.frombuffer(rec_b, emu_lib.RESULT_DTYPE)
    ops = np.frombuffer(ops_b, np.uint8)
    for i, (p, t) in enumerate(_real_pairs()):
        o = O.OracleAligner(3, [0, 4, 6, 2])
        o.set_alignment_scope(True)
        s = o.align_end2end(p, t)
        r = rec[i]
        got = ops[r["cigar_begin"]:r["cigar_begin"] + r["cigar_length"]].tobytes()
        assert (int(r["score"]), int(r["status"]), got) == (s, o.status(), o.cigar()[0]), i
