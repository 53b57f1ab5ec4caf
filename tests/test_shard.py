"""Multi-GPU sharding logic on CPU: the LPT partition and the gather of
per-rank results, with world_size 2 over gloo (the alignment itself is
stood in by a deterministic function of the pair, so no GPU is needed)."""
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
