"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Public datasets are not used: each configuration is a seeded stand-in with the
stated sizes and error model (seed = 0x5EED0000 + configuration index).  The
edit model follows the benchmark description: per position, independently
with probability p, a substitution (new base uniform over ACGT, so it may be
silent), an insertion (a random base, then the original) or a deletion (skip),
with equal odds.

Sequences are returned as one contiguous uint8 buffer plus offsets/lengths,
the batch layout the C-ABI takes.
"""
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
SEED_BASE = 0x5EED0000


class PairSet:
    """Pairs in one buffer: pattern i = buf[p_off[i]:p_off[i]+p_len[i]], text likewise."""

    def __init__(self, buf, p_off, p_len, t_off, t_len):
        self.buf = np.ascontiguousarray(buf, dtype=np.uint8)
        self.p_off = np.asarray(p_off, dtype=np.int64)
        self.p_len = np.asarray(p_len, dtype=np.int32)
        self.t_off = np.asarray(t_off, dtype=np.int64)
        self.t_len = np.asarray(t_len, dtype=np.int32)

    def __len__(self):
        return len(self.p_len)

    def pair(self, i):
        p = self.buf[self.p_off[i]:self.p_off[i] + self.p_len[i]].tobytes()
        t = self.buf[self.t_off[i]:self.t_off[i] + self.t_len[i]].tobytes()
        return p, t

    def subset(self, idx):
        idx = np.asarray(idx)
        return PairSet(self.buf, self.p_off[idx], self.p_len[idx], self.t_off[idx], self.t_len[idx])

    def cells(self):
        """Equivalent DP cells (sum of n*m)."""
        return int(np.sum(self.p_len.astype(np.int64) * self.t_len.astype(np.int64)))


def _mutate(rng, patterns, p_len, rate):
    """Apply the per-position sub/ins/del model; returns (flat texts, text lengths)."""
    total = len(patterns)
    pair_of = np.repeat(np.arange(len(p_len)), p_len)
    p = rate[pair_of]
    u = rng.random(total)
    op = rng.integers(0, 3, total)
    edit = u < p
    sub = edit & (op == 0)
    ins = edit & (op == 1)
    dele = edit & (op == 2)
    counts = np.ones(total, dtype=np.int64)
    counts[ins] = 2
    counts[dele] = 0
    src = np.repeat(np.arange(total), counts)
    out = patterns[src].copy()
    # First emitted char of an insertion is a random base; a substitution's
    # only char is a random base.
    first = np.ones(len(src), dtype=bool)
    first[1:] = src[1:] != src[:-1]
    rnd = ACGT[rng.integers(0, 4, len(src))]
    repl = (ins[src] & first) | sub[src]
    out[repl] = rnd[repl]
    t_len = np.bincount(pair_of, weights=counts, minlength=len(p_len)).astype(np.int32)
    return out, t_len


def _interleave(patterns, p_len, texts, t_len):
    n = len(p_len)
    p_end = np.cumsum(p_len.astype(np.int64))
    t_end = np.cumsum(t_len.astype(np.int64))
    p_start = p_end - p_len
    t_start = t_end - t_len
    pair_len = p_len.astype(np.int64) + t_len
    base = np.concatenate([[0], np.cumsum(pair_len)[:-1]])
    buf = np.empty(int(pair_len.sum()), dtype=np.uint8)
    # pattern i at base[i], text i right after it
    pos_p = np.repeat(base - p_start, p_len) + np.arange(len(patterns))
    pos_t = np.repeat(base + p_len - t_start, t_len) + np.arange(len(texts))
    buf[pos_p] = patterns
    buf[pos_t] = texts
    return PairSet(buf, base, p_len, base + p_len, t_len)


def uniform_pairs(num, len_lo, len_hi, rate_lo, rate_hi, seed):
    """Pattern length U[len_lo, len_hi], per-pair edit rate U[rate_lo, rate_hi]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p_len = rng.integers(len_lo, len_hi + 1, num).astype(np.int32)
    rate = rng.uniform(rate_lo, rate_hi, num) if rate_hi > rate_lo else np.full(num, rate_lo)
    patterns = ACGT[rng.integers(0, 4, int(p_len.sum()))]
    texts, t_len = _mutate(rng, patterns, p_len, rate)
    return _interleave(patterns, p_len, texts, t_len)


def pairs_with_lengths(p_len, rate, seed):
    """Patterns of the given lengths, texts by the per-position model at
    per-pair edit rates `rate`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p_len = np.asarray(p_len, dtype=np.int32)
    patterns = ACGT[rng.integers(0, 4, int(p_len.sum()))]
    texts, t_len = _mutate(rng, patterns, p_len, np.asarray(rate, dtype=np.float64))
    return _interleave(patterns, p_len, texts, t_len)


def config5(num, seed=SEED_BASE + 5):
    """Serving request mix: 70% 150 bp pairs at 2% edits, 25% log-uniform
    1-10 kbp at 8%, 5% 50 kbp at 10% (the per-position model), in a random
    arrival order.  Returns (PairSet, kind per request: 0 short, 1 medium,
    2 long)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kind = rng.choice(3, size=num, p=[0.70, 0.25, 0.05])
    p_len = np.where(kind == 0, 150,
                     np.where(kind == 1, np.exp(rng.uniform(np.log(1000), np.log(10000), num)), 50000))
    rate = np.choose(kind, [0.02, 0.08, 0.10])
    return pairs_with_lengths(p_len.astype(np.int32), rate, seed + 1), kind


def config1(num=10_000):
    """Plain method, small: n = 100, p = 0.05 (gap-affine 0,4,6,2 end-to-end)."""
    return uniform_pairs(num, 100, 100, 0.05, 0.05, SEED_BASE + 1)


def config2(num=1_000_000):
    """Short-read batch: n ~ U[100,150], p ~ U[0,0.04] per pair."""
    return uniform_pairs(num, 100, 150, 0.0, 0.04, SEED_BASE + 2)


def config4(num=200_000, seed=SEED_BASE + 4, chunk=10_000):
    """Ends-free / extension: core length U[500, 5000] at a 10% edit rate
    (the per-position sub/ins/del model), and every sequence (pattern and
    text, independently) flanked on each side by a random ACGT tail of
    U[0, 0.2 * core] bases.  Generated in chunks of `chunk` pairs (chunk i
    seeded with seed + i) to bound the memory of the generator."""
    parts = [_config4_chunk(min(chunk, num - i), seed + i // chunk) for i in range(0, num, chunk)]
    if len(parts) == 1:
        return parts[0]
    base = np.concatenate([[0], np.cumsum([len(q.buf) for q in parts])[:-1]]).astype(np.int64)
    return PairSet(np.concatenate([q.buf for q in parts]),
                   np.concatenate([q.p_off + b for q, b in zip(parts, base)]),
                   np.concatenate([q.p_len for q in parts]),
                   np.concatenate([q.t_off + b for q, b in zip(parts, base)]),
                   np.concatenate([q.t_len for q in parts]))


def _config4_chunk(num, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    core_len = rng.integers(500, 5001, num).astype(np.int32)
    cores = ACGT[rng.integers(0, 4, int(core_len.sum()))]
    texts, t_core = _mutate(rng, cores, core_len, np.full(num, 0.10))
    # Flank lengths: pattern left/right, text left/right.
    fl = (rng.random((num, 4)) * (0.2 * core_len[:, None] + 1)).astype(np.int64)
    fl = np.minimum(fl, (0.2 * core_len[:, None]).astype(np.int64))
    p_len = (core_len + fl[:, 0] + fl[:, 1]).astype(np.int32)
    t_len = (t_core + fl[:, 2] + fl[:, 3]).astype(np.int32)
    total = int(p_len.sum()) + int(t_len.sum())
    rnd = ACGT[rng.integers(0, 4, total)]  # flank bases (cores overwrite their part)
    p_off = np.concatenate([[0], np.cumsum(p_len.astype(np.int64) + t_len)[:-1]]).astype(np.int64)
    t_off = p_off + p_len
    buf = rnd.copy()
    c_start = np.concatenate([[0], np.cumsum(core_len.astype(np.int64))[:-1]])
    t_start = np.concatenate([[0], np.cumsum(t_core.astype(np.int64))[:-1]])
    pos_p = np.repeat(p_off + fl[:, 0] - c_start, core_len) + np.arange(int(core_len.sum()))
    pos_t = np.repeat(t_off + fl[:, 2] - t_start, t_core) + np.arange(int(t_core.sum()))
    buf[pos_p] = cores
    buf[pos_t] = texts
    return PairSet(buf, p_off, p_len, t_off, t_len)


def pack2bits(ps):
    """2-bit pack every sequence of a PairSet (A0 C1 G2 T3, LSB-first, 16 bases
    per 32-bit word; the byte order equals the reference's 4-per-byte packing,
    src/sequences.rs:55-74).  Each sequence starts on a word boundary.

    Returns (words uint32[], p_word_off, t_word_off)."""
    code = np.zeros(256, dtype=np.uint8)
    code[ord("C")] = 1; code[ord("G")] = 2; code[ord("T")] = 3
    code[ord("c")] = 1; code[ord("g")] = 2; code[ord("t")] = 3
    n = len(ps)
    lens = np.empty(2 * n, dtype=np.int64)
    lens[0::2] = ps.p_len
    lens[1::2] = ps.t_len
    offs = np.empty(2 * n, dtype=np.int64)
    offs[0::2] = ps.p_off
    offs[1::2] = ps.t_off
    words = (lens + 15) // 16
    woff = np.concatenate([[0], np.cumsum(words)[:-1]])
    total_words = int(words.sum())
    out = np.zeros(total_words * 16, dtype=np.uint8)
    dst = np.repeat(woff * 16 - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) + np.arange(int(lens.sum()))
    src = np.repeat(offs - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) + np.arange(int(lens.sum()))
    out[dst] = code[ps.buf[src]]
    q = out.reshape(-1, 16).astype(np.uint32)
    shifts = (2 * np.arange(16, dtype=np.uint32))
    packed = np.bitwise_or.reduce(q << shifts, axis=1).astype(np.uint32)
    return packed, woff[0::2].astype(np.int64), woff[1::2].astype(np.int64)


def config3(num=20_000, seed=SEED_BASE + 3):
    """Uneven long reads: n log-uniform in [1 kbp, 20 kbp], per-pair edit rate
    U[0.05, 0.15]; 40% substitutions, 30% insertions and 30% deletions, indel
    lengths geometric with mean 3.  (Gap-affine 2-piece, BiWFA.)"""
    rng = np.random.Generator(np.random.PCG64(seed))
    p_len = np.exp(rng.uniform(np.log(1000), np.log(20000), num)).astype(np.int32)
    rate = rng.uniform(0.05, 0.15, num)
    total = int(p_len.sum())
    patterns = ACGT[rng.integers(0, 4, total)]
    pair_of = np.repeat(np.arange(num), p_len)
    starts = np.concatenate([[0], np.cumsum(p_len)[:-1]])
    pair_end = (starts + p_len)[pair_of]
    u = rng.random(total)
    edit = u < rate[pair_of]
    kind = rng.random(total)
    sub = edit & (kind < 0.4)
    ins = edit & (kind >= 0.4) & (kind < 0.7)
    dele = edit & (kind >= 0.7)
    glen = rng.geometric(1.0 / 3.0, total)
    pos = np.arange(total)
    # A deletion at i removes i .. i+len-1 (within its pair).
    end = np.where(dele, np.minimum(pos + glen, pair_end), -1)
    deleted = np.maximum.accumulate(end) > pos
    keep = ~deleted
    counts = np.where(keep, np.where(ins, glen + 1, 1), 0).astype(np.int64)
    src = np.repeat(pos, counts)
    out = patterns[src].copy()
    last = np.ones(len(src), dtype=bool)
    last[:-1] = src[1:] != src[:-1]
    rnd = ACGT[rng.integers(0, 4, len(src))]
    repl = (ins[src] & ~last) | sub[src]
    out[repl] = rnd[repl]
    t_len = np.bincount(pair_of, weights=counts, minlength=num).astype(np.int32)
    return _interleave(patterns, p_len, out, t_len)
