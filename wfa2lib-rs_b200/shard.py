"""Multi-GPU replicas: pairs are independent, so a batch shards across GPUs
with no collective on the alignment path (one process per GPU).

The pairs are dealt to ranks longest-expected-first onto the least-loaded
rank (LPT), with the expected cost of a pair taken as (n + m)^2 (the
wavefront work grows with the square of the score, which grows with the
lengths).  Each rank aligns its shard into its own result buffer; one gather
at the end returns every result to rank 0 in input order.
"""
import heapq

import numpy as np


def expected_cost(p_len, t_len):
    s = np.asarray(p_len, dtype=np.int64) + np.asarray(t_len, dtype=np.int64)
    return s * s


def lpt_partition(cost, world):
    """Index arrays, one per rank: pairs in order of decreasing cost (ties by
    index), each to the rank with the least assigned cost so far (ties by
    rank).  Deterministic, so every rank computes the same partition."""
    cost = np.asarray(cost, dtype=np.int64)
    order = np.lexsort((np.arange(len(cost)), -cost))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(i))
        heapq.heappush(heap, (load + int(cost[i]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def run_sharded(align_fn, p_len, t_len, rank, world, group=None):
    """Align this rank's shard with align_fn(indices) -> numpy structured
    array (one record per index) and gather all records to rank 0 in input
    order (None on the other ranks).  With world == 1 no process group is
    needed."""
    shards = lpt_partition(expected_cost(p_len, t_len), world)
    mine = shards[rank]
    local = align_fn(mine)
    if world == 1:
        return local
    import torch.distributed as dist
    gathered = [None] * world if rank == 0 else None
    dist.gather_object((mine, local), gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = np.empty(len(p_len), dtype=local.dtype)
    for idx, rec in gathered:
        out[idx] = rec
    return out
