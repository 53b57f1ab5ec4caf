"""Multi-GPU replicas: pairs are independent, so a batch shards across GPUs
with no collective on the alignment path (one process per GPU).

The pairs are dealt to ranks longest-expected-first onto the least-loaded
rank (LPT), with the expected cost of a pair taken as (n + m)^2 (the
wavefront work grows with the square of the score, which grows with the
lengths).  Each rank aligns its shard into its own result buffer; one gather
at the end returns every result, with its CIGAR bytes, to rank 0 in input
order.
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


def _ragged_copy(dst, dst_begin, src, src_begin, length, chunk=1 << 16):
    """dst[dst_begin[i]:+length[i]] = src[src_begin[i]:+length[i]] for every
    i, vectorised over chunks of pairs."""
    for a in range(0, len(length), chunk):
        ln = length[a:a + chunk].astype(np.int64)
        tot = int(ln.sum())
        if tot == 0:
            continue
        start = np.concatenate([[0], np.cumsum(ln)[:-1]])
        within = np.arange(tot, dtype=np.int64) - np.repeat(start, ln)
        dst[np.repeat(dst_begin[a:a + chunk], ln) + within] = src[np.repeat(src_begin[a:a + chunk], ln) + within]


def assemble(parts, n):
    """Records in input order from (indices, records, CIGAR bytes or None)
    per rank.  With CIGARs, the records' cigar_begin/cigar_length index the
    rank's bytes; the result packs them densely in input order and rewrites
    cigar_begin to index the returned buffer."""
    dtype = parts[0][1].dtype
    out = np.empty(n, dtype=dtype)
    for idx, rec, _ in parts:
        out[idx] = rec
    if parts[0][2] is None:
        return out
    lens = out["cigar_length"].astype(np.int64)
    dense_begin = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    ops = np.empty(int(lens.sum()), dtype=np.uint8)
    for idx, rec, src in parts:
        _ragged_copy(ops, dense_begin[idx], src, rec["cigar_begin"].astype(np.int64),
                     rec["cigar_length"])
    out["cigar_begin"] = dense_begin.astype(out["cigar_begin"].dtype)
    return out, ops


def run_sharded(align_fn, p_len, t_len, rank, world, group=None):
    """Align this rank's shard and gather every result to rank 0 in input
    order (None on the other ranks).  align_fn(indices) returns either a
    numpy structured array (one record per index) or (records, CIGAR bytes)
    with records holding cigar_begin / cigar_length into those bytes; in the
    second case rank 0 gets (records, packed CIGAR bytes).  With world == 1
    no process group is needed."""
    shards = lpt_partition(expected_cost(p_len, t_len), world)
    mine = shards[rank]
    local = align_fn(mine)
    rec, ops = local if isinstance(local, tuple) else (local, None)
    if world == 1:
        parts = [(mine, rec, ops)]
    else:
        import torch.distributed as dist
        parts = [None] * world if rank == 0 else None
        dist.gather_object((mine, rec, ops), parts, dst=0, group=group)
        if rank != 0:
            return None
    return assemble(parts, len(p_len))
