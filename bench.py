"""Benchmark: short-read batch (1,000,000 pairs, 100-150 bp, 0-4% edits,
2-bit packed), gap-affine (0,4,6,2), end-to-end, score + CIGAR.  Other
workloads (`--workload small|longread`): 10,000 x 100 bp pairs at 5% edits,
and an uneven long-read batch (1-20 kbp, 5-15% edits, gap-affine 2-piece,
BiWFA).

A step is one batched alignment of the whole pair set.  `value` is pairs/s
with inputs resident in HBM (device-buffer API, CUDA events on the launching
stream); `e2e` is the same metric through the host-buffer API, with the
host->device input copies and device->host result/CIGAR copies inside every
step.  Roofline: the HBM algorithmic bytes of the workload (packed inputs, an
8-byte score/status record and one byte per CIGAR op per pair) over the
alignment kernel's event-timed duration.  Between timed steps L2 is flushed
by writing a 512 MiB buffer (outside the per-step events).

`--impl reference` times the CPU restatement of the reference path (the
oracle; no Rust toolchain exists on the box) with all host threads on the
same pairs.  Multi-GPU: one process per GPU, each aligning its own seeded
shard of the same size (weak scaling, no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))
PEN = [0, 4, 6, 2]
METRIC = "pairs/sec + equiv GCUPS, batched vs plain GPU (bit-exact); served p50/p99 ms"
WORKLOAD = "short-read batch: 1,000,000 pairs, n~U[100,150], p~U[0,0.04], 2-bit packed, gap-affine 0,4,6,2, end-to-end, score+CIGAR"


def load_pkg():
    from _pkg import load
    return load()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# Workloads: (description, generator, metric, penalties, span, oracle mode,
# heuristic (kind, params), packed).  span: 0 align_end2end, 1 align_endsfree
# (here the extension span), 2 BiWFA (align_biwfa); oracle mode likewise.
WORKLOADS = {
    "shortread": (WORKLOAD, "short", 3, [0, 4, 6, 2], 0, 0, (0, ()), True),
    "small": ("plain method, small: 10,000 x 100 bp, p=0.05, gap-affine 0,4,6,2, end-to-end, "
              "score+CIGAR (2-bit packed)", "small", 3, [0, 4, 6, 2], 0, 0, (0, ()), True),
    "longread": ("uneven long-read batch: 20,000 pairs, n log-uniform [1,20] kbp, p~U[0.05,0.15], "
                 "60% indels (geometric, mean 3), gap-affine 2-piece 0,4,6,2,24,1, BiWFA, CIGAR "
                 "(2-bit packed)", "long", 4, [0, 4, 6, 2, 24, 1], 2, 2, (0, ()), True),
    "extension": ("ends-free / extension batch: 200,000 pairs, core U[500,5000] bp at 10% edits, "
                  "random flanks of U[0, 0.2 core] on every end, gap-affine 0,4,6,2, extension span, "
                  "X-drop 200 (cutoff every step), score+CIGAR (ASCII)", "c4", 3, [0, 4, 6, 2], 1,
                  1, (2, (200, 1, 0)), False),
}


def make_workload(num_pairs, rank, kind="short", packed=True, length_range=None):
    """(pkg, synth, pairs, sequence buffer, pattern offsets, text offsets) in
    the batch layout: 2-bit words and word offsets, or bytes and byte offsets."""
    pkg = load_pkg()
    from wfa_b200 import synth
    if kind == "short":
        ps = synth.uniform_pairs(num_pairs, 100, 150, 0.0, 0.04, synth.SEED_BASE + 2 + 1000 * rank)
    elif kind == "small":
        ps = synth.uniform_pairs(num_pairs, 100, 100, 0.05, 0.05, synth.SEED_BASE + 1 + 1000 * rank)
    elif kind == "c4":
        ps = synth.config4(num_pairs, synth.SEED_BASE + 4 + 1000 * rank)
    else:
        ps = synth.config3(num_pairs, synth.SEED_BASE + 3 + 1000 * rank)
    if length_range:
        # Only the pairs of one pattern-length class, drawn from a pool eight
        # times larger (for profiling one class on a capture-sized case).
        lo, hi = length_range
        pool = synth.config3(8 * num_pairs, synth.SEED_BASE + 3 + 1000 * rank) if kind == "long" else ps
        keep = np.where((pool.p_len >= lo) & (pool.p_len <= hi))[0][:num_pairs]
        ps = pool.subset(keep)
    if not packed:
        return pkg, synth, ps, np.concatenate([ps.buf, np.zeros(16, np.uint8)]), ps.p_off, ps.t_off
    words, pwo, two = synth.pack2bits(ps)
    words = np.concatenate([words, np.zeros(4, np.uint32)])
    return pkg, synth, ps, words, pwo, two


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dram_traffic(kind, pairs):
    """DRAM bytes (read + write) of one alignment launch over `pairs` pairs,
    scaled from the per-pair figure of the workload's ncu capture, whose
    summary (command and numbers) is in profiles/; None without one."""
    path = os.path.join(ROOT, "profiles", f"dram_bytes_per_pair_{kind}.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_pair"):
                    return float(line.split()[1]) * pairs
    except OSError:
        pass
    return None


def profile_figure(name, kind):
    """A per-pair figure of the workload's ncu capture (profiles/<name>_<kind>.txt,
    a line `<name> <value>`), or None without one."""
    path = os.path.join(ROOT, "profiles", f"{name}_{kind}.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(name):
                    return float(line.split()[1])
    except OSError:
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(ps, threads, max_pairs=None, metric=3, pen=PEN, mode=0, heur=(0, ())):
    """The oracle (C++ restatement) on the host cores; returns (pairs/s, pairs, secs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n = len(ps) if max_pairs is None else min(len(ps), max_pairs)
    sub = ps.subset(np.arange(n))
    hp = tuple(heur[1]) + (0, 0, 0)
    secs, _, _, _ = O.batch(metric, pen, ps.buf.tobytes(), sub.p_off, sub.p_len, sub.t_off,
                            sub.t_len, compute_alignment=True, mode=mode, heuristic=heur[0],
                            hparams=hp[:3], threads=threads, want_results=False)
    return n / secs, n, secs


# Shared-memory bytes per computed cell of each metric's compute step
# (reads + writes of 4-byte offsets): edit 4, indel 3, linear 4, affine 8,
# affine 2-piece 14; indexed by the oracle's metric number.
CELL_RW = {0: 3, 1: 4, 2: 4, 3: 8, 4: 14}


def oracle_check(ps, n_check, metric, pen, omode, heur, threads, checks):
    """Scores, statuses and CIGARs (FNV-1a hashes) of the first n_check pairs
    against the oracle, outside every timed region.  checks: name ->
    (result records, CIGAR byte buffer, begin offset of each pair's CIGAR in
    it).  Returns ({name: mismatching pairs}, the oracle's work sums over
    those pairs: cells computed, bases compared, CIGAR ops)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sub = ps.subset(np.arange(n_check))
    hp = tuple(heur[1]) + (0, 0, 0)
    work = np.zeros(3, np.int64)
    _, sc, st, hs = O.batch(metric, pen, ps.buf.tobytes(), sub.p_off, sub.p_len, sub.t_off,
                            sub.t_len, compute_alignment=True, mode=omode, heuristic=heur[0],
                            hparams=hp[:3], threads=threads, want_results=True, work=work)
    out = {}
    for name, (rec, ops, begin) in checks.items():
        r = rec[:n_check]
        gh = O.hash_ops(ops, begin[:n_check], r["cigar_length"], threads)
        bad = (r["score"] != sc) | (r["status"] != st) | (gh != hs)
        out[name] = int(bad.sum())
    return out, work


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    desc, kind, metric, pen, span, omode, heur, packed = WORKLOADS[args.workload]
    pkg, synth, ps, _, _, _ = make_workload(args.pairs, 0, kind, packed=False)
    threads = os.cpu_count() or 1
    sample = min(len(ps), args.cpu_sample)
    for _ in range(args.warmup):
        cpu_baseline(ps, threads, max_pairs=min(sample, 2 * threads), metric=metric, pen=pen, mode=omode,
                     heur=heur)
    tot_secs, tot_pairs = 0.0, 0
    for _ in range(args.steps):
        rate, n, secs = cpu_baseline(ps, threads, max_pairs=sample, metric=metric, pen=pen, mode=omode,
                                     heur=heur)
        tot_secs += secs
        tot_pairs += n
    value = tot_pairs / tot_secs
    cells = float(np.mean(ps.p_len.astype(np.float64) * ps.t_len))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * tot_secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
            "config": {"workload": desc, "sample_pairs_per_step": sample},
            "gcups": value * cells / 1e9,
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                             "sample": f"{sample} pairs of the workload per step"},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_gpu(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    desc, kind, metric, pen, span, omode, heur, packed = WORKLOADS[args.workload]
    pkg, synth, ps, words, pwo, two = make_workload(args.pairs, rank, kind, packed,
                                                    args.length_range)
    n = len(ps)
    a = pkg.WavefrontAligner(metric, pen, device=local)
    a.set_alignment_scope(True)
    if args.lanes:
        a.set_lanes_per_pair(args.lanes)
    if args.bi_lanes:
        a.set_biwfa_lanes(args.bi_lanes)
    if span == 1:
        a.set_alignment_extension()
    if heur[0]:
        a.set_heuristic(heur[0], *heur[1])
    wbytes = words.view(np.uint8)

    # Device-resident inputs and outputs.
    t_words = torch.from_numpy(wbytes).to(dev)
    t_po, t_pl = torch.from_numpy(pwo).to(dev), torch.from_numpy(ps.p_len).to(dev)
    t_to, t_tl = torch.from_numpy(two).to(dev), torch.from_numpy(ps.t_len).to(dev)
    caps = 2 * (ps.p_len.astype(np.int64) + ps.t_len) + 1
    coff = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
    t_co = torch.from_numpy(coff).to(dev)
    cig = torch.empty(int(caps.sum()) + 16, dtype=torch.uint8, device=dev)
    res = torch.empty(n * 10, dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        a.align_batch_device(t_words.data_ptr(), t_words.numel(), t_po.data_ptr(),
                             t_pl.data_ptr(), t_to.data_ptr(), t_tl.data_ptr(), n, res.data_ptr(),
                             cig.data_ptr(), t_co.data_ptr(), int(caps.sum()), packed=packed,
                             span=span, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = a.kernel_launches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms, kern_ms = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            kern_ms.append(a.last_kernel_ms())
    torch.cuda.synchronize()
    launches = a.kernel_launches() - launches0
    reruns = a.last_rerun_pairs()
    lanes = a.last_lanes_per_pair()
    from wfa_b200.aligner import autotune_report
    tuned = [ln for ln in autotune_report().splitlines() if ln]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * n * args.steps / (total_ms / 1000.0)

    # Results of the last step (for the byte counts and a parity spot check).
    rd = res.cpu().numpy().view(pkg.RESULT_DTYPE)
    assert np.all((rd["status"] >= 0) & (rd["status"] < 100)), "a pair was left unaligned"
    cig_ops = int(rd["cigar_length"].astype(np.int64).sum())
    if packed:
        in_bytes = int(((ps.p_len + 3) // 4).sum() + ((ps.t_len + 3) // 4).sum())
    else:
        in_bytes = int(ps.p_len.astype(np.int64).sum() + ps.t_len.astype(np.int64).sum())
    alg_bytes = in_bytes + 8 * n + cig_ops
    kms = float(np.mean(kern_ms))
    hbm_peak, peak_kind = peaks()
    achieved = alg_bytes / (kms / 1000.0) / 1e9
    cells = float(np.sum(ps.p_len.astype(np.float64) * ps.t_len))

    if args.no_e2e:
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
                "ms_per_step": total_ms / args.steps, "kernel_ms": kms, "gpu_launches": int(launches),
                "roofline_achieved_gbs": achieved, "lanes_per_pair": lanes,
                "rerun_pairs_per_step": int(reruns), "autotune": tuned}
        if rank == 0:
            print(json.dumps(line), flush=True)
        a.close()
        return

    # End to end: host (pinned) buffers through the host-buffer API.
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    h_words, h_po, h_pl, h_to, h_tl = pin(words), pin(pwo), pin(ps.p_len), pin(two), pin(ps.t_len)
    h_res = torch.zeros(n * 10, dtype=torch.int32).pin_memory().numpy().view(pkg.RESULT_DTYPE)
    h_cig = torch.zeros(int(caps.sum()) + 16, dtype=torch.uint8).pin_memory().numpy()
    e2e_ms = []
    # Long workloads (tens of seconds a step) time the host-buffer form once,
    # after one untimed run.
    e2e_warm, e2e_steps = (1, 1) if args.workload == "longread" else (args.warmup, args.steps)
    for i in range(e2e_warm + e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hr, hc = a.align_batch(h_words, h_po, h_pl, h_to, h_tl, packed=packed, out_results=h_res,
                               out_cigars=h_cig, span=span)
        t1 = time.perf_counter()
        if i >= e2e_warm:
            e2e_ms.append((t1 - t0) * 1000)
    e2e_kernel_ms = a.last_kernel_ms()
    e2e_reruns = a.last_rerun_pairs()
    e2e_lanes = a.last_lanes_per_pair()
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * n * e2e_steps / (e2e_total / 1000.0)
    assert np.array_equal(hr["score"], rd["score"])
    h2d = int(h_words.nbytes + h_po.nbytes + h_pl.nbytes + h_to.nbytes + h_tl.nbytes)
    d2h = int(hr.nbytes + int(hr["cigar_length"].astype(np.int64).sum()))

    # Plain per-call form: one pair per call (host buffers), on a sample.
    plain_n = min(args.plain_pairs, n)
    raw = [ps.pair(i) for i in range(plain_n)]
    plain = {0: a.align_end2end, 1: a.align_endsfree, 2: a.align_biwfa}[span]
    for p, t in raw[:min(50, plain_n)]:
        plain(p, t)
    t0 = time.perf_counter()
    for p, t in raw:
        plain(p, t)
    plain_secs = time.perf_counter() - t0
    plain_value = plain_n / plain_secs

    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)",
            "config": {"workload": desc, "pairs_per_gpu": n, "l2": "flushed (512 MiB write) between steps",
                       "form": "batched persistent kernel, device-resident inputs"},
            "gcups": world * cells * args.steps / (total_ms / 1000.0) / 1e9,
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "api": "wfa_batch_align (pinned host buffers)",
                    "steps": e2e_steps, "kernel_ms": e2e_kernel_ms, "rerun_pairs": int(e2e_reruns),
                    "lanes_per_pair": e2e_lanes},
            "plain": {"value": plain_value, "unit": "pairs/s", "pairs": plain_n,
                      "api": {0: "wfa_align_end2end", 1: "wfa_align_endsfree",
                              2: "wfa_align_biwfa"}[span] + ", one pair per call"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": dram_traffic(args.workload, n),
                         "peak_kind": peak_kind,
                         "kernel_ms": kms, "algorithmic_bytes_per_launch": alg_bytes},
            "gpu_launches": int(launches),
            "rerun_pairs_per_step": int(reruns),
            "lanes_per_pair": lanes, "autotune": tuned,
            "clocks": clk.summary()}
    # The alignment kernel is bound by instruction issue: warp instructions
    # per pair (ncu) x pairs/s against 4 schedulers x SMs x the sampled clock.
    ipp = profile_figure("warp_inst_per_pair", args.workload)
    if ipp is not None:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = line["clocks"].get("sm_mhz") or 1965.0
        issue_peak = 4 * sms * mhz * 1e6
        issue = value / world * ipp
        line["roofline_issue"] = {"bound": "issue", "achieved": issue, "peak": issue_peak,
                                  "unit": "warp-inst/s", "frac": issue / issue_peak,
                                  "warp_inst_per_pair": ipp}
    if rank == 0 and not args.no_parity:
        # Every checked pair against the oracle: the last timed device step's
        # slots and the last host-buffer call's packed CIGARs.
        threads = os.cpu_count() or 1
        n_check = min(n, args.parity_pairs)
        dev_cig = cig.cpu().numpy()
        checks = {"device": (rd, dev_cig, coff + rd["cigar_begin"]),
                  "e2e": (hr, hc, hr["cigar_begin"].astype(np.int64))}
        bad, work = oracle_check(ps, n_check, metric, pen, omode, heur, threads, checks)
        line["parity"] = {"pairs_checked": n_check, "mismatches": bad["device"],
                          "e2e_mismatches": bad["e2e"], "oracle": "port (C++ restatement)",
                          "fields": "score, status, CIGAR bytes (FNV-1a 64 per pair)"}
        # Shared-memory roofline (on-chip wavefront traffic): per pair
        # C x 4 B x (R + W) + 2 ceil(X / 4) + 4 L from the oracle's work
        # counters, scaled to the whole launch; peak = SMs x 128 B/clk x
        # the sampled SM clock.
        scale = n / n_check
        cells, bases, ops = (float(x) * scale for x in work)
        smem_bytes = cells * 4 * CELL_RW[metric] + 2 * np.ceil(bases / 4) + 4 * ops
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = line["clocks"].get("sm_mhz") or 1965.0
        smem_peak = sms * 128 * mhz * 1e6 / 1e9
        smem_ach = smem_bytes / (kms / 1000.0) / 1e9
        line["roofline_smem"] = {"bound": "smem", "achieved": smem_ach, "peak": smem_peak,
                                 "unit": "GB/s", "frac": smem_ach / smem_peak,
                                 "bytes_per_pair": smem_bytes / n,
                                 "peak_kind": f"{sms} SMs x 128 B/clk x sampled {mhz:.0f} MHz",
                                 "work_per_pair": {"cells": cells / n, "bases": bases / n,
                                                   "cigar_ops": ops / n}}
        bound_hbm = hbm_peak * 1e9 / (alg_bytes / n)
        bound_smem = smem_peak * 1e9 / (smem_bytes / n)
        lim = "hbm" if bound_hbm < bound_smem else "smem"
        line["roofline_memory"] = {"limit": lim, "pairs_per_s_bound": min(bound_hbm, bound_smem),
                                   "frac": value / world / min(bound_hbm, bound_smem)}
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, m, secs = cpu_baseline(ps, threads, max_pairs=args.cpu_sample, metric=metric, pen=pen,
                                     mode=omode, heur=heur)
        line["cpu_baseline"] = {"value": rate, "unit": "pairs/s", "cores": threads, "kind": "port",
                                "sample": f"first {m} pairs of the workload ({secs:.2f} s wall)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    a.close()
    if world > 1:
        torch.distributed.destroy_process_group()


SERVE = ("serving: open-loop Poisson arrivals, request mix 70% 150 bp at 2%, 25% log-uniform "
         "1-10 kbp at 8%, 5% 50 kbp at 10% edits, gap-affine 0,4,6,2, CIGAR; high-memory "
         "end-to-end, BiWFA above a 256 MiB predicted footprint")


def run_serve(args):
    """Open-loop serving sweep: requests arrive as a Poisson process at each
    rate; latency is submit -> result ready (the server's clock); throughput
    is requests completed over the span from the first arrival to the last
    result.  Rank 0 only (one server per GPU)."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    pkg = load_pkg()
    from wfa_b200 import synth
    rates = [float(x) for x in args.rates.split(",")]
    per_rate = args.pairs
    srv = pkg.Server(pkg.GAP_AFFINE, PEN, device=local, workers=args.workers,
                     short_workers=args.workers, biwfa_workers=args.workers,
                     max_batch_bytes=16 << 30, resident=args.resident)
    # Warm-up: a few requests of each kind.
    wps, _ = synth.config5(64, synth.SEED_BASE + 55)
    for i in range(len(wps)):
        srv.submit(*wps.pair(i))
    left = len(wps)
    while left:
        left -= len(srv.poll(timeout_ms=500))
    table = []
    for j, lam in enumerate(rates):
        ps, kind = synth.config5(per_rate, synth.SEED_BASE + 5 + 1000 * j)
        reqs = [ps.pair(i) for i in range(len(ps))]
        rng = np.random.default_rng(j)
        arrive = np.cumsum(rng.exponential(1.0 / lam, len(reqs)))
        recs = {}
        stop = threading.Event()

        def poller():
            while True:
                for r in srv.poll(timeout_ms=50):
                    recs[r["id"]] = (r, time.perf_counter())
                if stop.is_set() and len(recs) >= len(reqs):
                    break

        th = threading.Thread(target=poller, daemon=True)
        th.start()
        ids = []
        t0 = time.perf_counter()
        with ClockSampler(local) as clk:
            for i, (p, t) in enumerate(reqs):
                wait = t0 + arrive[i] - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                ids.append(srv.submit(p, t))
            stop.set()
            th.join()
        t_end = max(v[1] for v in recs.values())
        lat = np.array([recs[i][0]["latency_ns"] for i in ids]) / 1e6
        kinds = np.asarray(kind)
        bad = [i for i in ids if recs[i][0]["status"] < 0]
        assert not bad, f"requests failed: {srv.last_error()}"
        pct = lambda q, sel: float(np.percentile(lat[sel], q)) if np.any(sel) else None
        row = {"rate_req_s": lam, "requests": len(reqs),
               "throughput_req_s": len(reqs) / (t_end - t0),
               "p50_ms": pct(50, kinds >= 0), "p99_ms": pct(99, kinds >= 0),
               "p50_ms_by_kind": [pct(50, kinds == k) for k in range(3)],
               "p99_ms_by_kind": [pct(99, kinds == k) for k in range(3)],
               "biwfa_requests": int(sum(recs[i][0]["mode"] for i in ids)),
               "clocks": clk.summary()}
        table.append(row)
    srv.stop()
    best = max(table, key=lambda r: r["throughput_req_s"])
    line = {"metric": METRIC, "value": best["throughput_req_s"], "unit": "requests/s",
            "n_gpus": 1, "steps": len(rates), "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
            "config": {"workload": SERVE, "requests_per_rate": per_rate,
                       "workers_per_lane": args.workers, "lanes": "short (n+m<=1024), long, BiWFA",
                       "short_lane": "resident stream" if args.resident else "host-buffer batches",
                       "form": "wfa_server_* continuous batching, host request buffers"},
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "sweep": table}
    print(json.dumps(line), flush=True)


STREAM = ("resident stream: short-read requests (n~U[100,150], p~U[0,0.04], ASCII, gap-affine "
          "0,4,6,2, end-to-end, score+CIGAR) submitted open loop in bursts every 0.2 ms at each "
          "offered rate to one persistent kernel (wfa_stream_*)")


def stream_rate(st, lam, seconds, seq, po, pl, to, tl, local, burst=0):
    """One offered rate (or, with burst, `burst` requests submitted at once
    in chunks as the ring frees): every wait is bounded by a deadline, and a
    rate the stream cannot keep up with reports what it completed."""
    n = len(pl)
    total = burst if burst else int(lam * seconds)
    chunk = 16384
    lat, done, errs = [], [0], []
    t0 = time.perf_counter()
    deadline = t0 + 3 * seconds + 30

    def poller():
        try:
            while done[0] < total and time.perf_counter() < deadline:
                recs, _ = st.poll_arrays(timeout_ms=5)
                if len(recs):
                    lat.append(recs["latency_ns"].copy())
                    if (recs["status"] < 0).any():
                        errs.append("failed request")
                    done[0] += len(recs)
        except Exception as e:  # reported below
            errs.append(repr(e))

    th = threading.Thread(target=poller, daemon=True)
    th.start()
    sent, busy = 0, 0
    with ClockSampler(local) as clk:
        while sent < total and time.perf_counter() < deadline and not errs:
            due = total if burst else min(total, int((time.perf_counter() - t0) * lam) + 1)
            k = min(due - sent, chunk)
            if k > 0:
                idx = np.arange(sent, sent + k) % n
                r = st.submit_many(seq, po[idx], pl[idx], to[idx], tl[idx])
                if r == -7:
                    busy += 1
                else:
                    sent += k
            time.sleep(0.0002)
        th.join(timeout=max(1.0, deadline - time.perf_counter()))
    t_end = time.perf_counter()
    assert not errs, errs
    lat_ms = np.concatenate(lat) / 1e6 if lat else np.zeros(1)
    return {"offered_req_s": None if burst else lam, "burst": burst or None, "requests": total,
            "submitted": sent, "completed": done[0], "throughput_req_s": done[0] / (t_end - t0),
            "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "busy_retries": busy, "clocks": clk.summary()}


def run_stream(args):
    """Open-loop sweep of the resident stream: at each offered rate a
    submitting thread hands the stream the requests due every 0.2 ms (one
    submit_many call, each pair still its own request) and a polling thread
    collects results; latency is submit to the poll that found the result
    (the library's clock).  Rank 0 only."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    pkg = load_pkg()
    from wfa_b200 import synth
    pool = synth.uniform_pairs(args.pairs, 100, 150, 0.0, 0.04, synth.SEED_BASE + 2)
    seq, po, pl, to, tl = pool.buf, pool.p_off, pool.p_len, pool.t_off, pool.t_len
    n = len(pool)
    st = pkg.Stream(pkg.GAP_AFFINE, PEN, device=local, max_len_sum=320, capacity=1 << 18)
    # Warm-up: the pool once.
    st.submit_many(seq, po[:min(n, 1 << 17)], pl[:min(n, 1 << 17)], to[:min(n, 1 << 17)],
                   tl[:min(n, 1 << 17)])
    def drain(limit_s):
        t_lim = time.perf_counter() + limit_s
        while st.pending() and time.perf_counter() < t_lim:
            st.poll_arrays(timeout_ms=50)
        assert st.pending() == 0, "the stream did not drain"

    drain(60)
    rates = [float(x) for x in args.rates.split(",")]
    table = []
    for lam in rates:
        table.append(stream_rate(st, lam, args.seconds, seq, po, pl, to, tl, local))
        print(json.dumps(table[-1]), file=sys.stderr, flush=True)
        drain(60)
    # Capacity: one burst of the whole pool at once.
    table.append(stream_rate(st, float("inf"), args.seconds, seq, po, pl, to, tl, local, burst=n))
    print(json.dumps(table[-1]), file=sys.stderr, flush=True)
    drain(60)
    stats = st.stats()
    st.stop()
    # The highest offered rate the stream kept up with (throughput within 5 %).
    kept = [r for r in table if r["offered_req_s"] and r["completed"] == r["requests"]
            and r["throughput_req_s"] >= 0.95 * r["offered_req_s"]] or table[:1]
    best = max(kept, key=lambda r: r["throughput_req_s"])
    line = {"metric": METRIC, "value": best["throughput_req_s"], "unit": "requests/s",
            "n_gpus": 1, "steps": len(rates), "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
            "config": {"workload": STREAM, "pool_pairs": n, "seconds_per_rate": args.seconds,
                       "form": "wfa_stream_* resident kernel, host request buffers (mapped)"},
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "stream": stats, "sweep": table}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="shortread", choices=sorted(WORKLOADS) + ["serve", "stream"])
    ap.add_argument("--seconds", type=float, default=1.0, help="stream: seconds per offered rate")
    ap.add_argument("--rates", default="50,200,800", help="serve: arrival rates (requests/s)")
    ap.add_argument("--length-range", default=None,
                    type=lambda s: tuple(int(x) for x in s.split(",")),
                    help="lo,hi: keep only pairs with pattern length in [lo, hi] (profiling)")
    ap.add_argument("--workers", type=int, default=2, help="serve: workers per lane")
    ap.add_argument("--resident", action="store_true",
                    help="serve: the short lane is a resident stream (wfa_stream_*)")
    ap.add_argument("--pairs", type=int, default=None)
    ap.add_argument("--plain-pairs", type=int, default=None)
    ap.add_argument("--cpu-sample", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--parity-pairs", type=int, default=None,
                    help="pairs checked against the oracle after the timed region")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--bi-lanes", type=int, default=0,
                    help="BiWFA lanes per pair (32, 128, 256, 512); 0: by length")
    ap.add_argument("--lanes", type=int, default=0,
                    help="lanes per pair (8, 16, 32); 0: autotuned")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer and plain forms")
    args = ap.parse_args()
    if args.workload == "stream":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the stream sweep measures the GPU request loop; the CPU arm is "
                              "timed on the batch workloads"}), flush=True)
            return
        args.pairs = 1 << 20 if args.pairs is None else args.pairs
        args.rates = "1e5,3e5,1e6,3e6" if args.rates == "50,200,800" else args.rates
        run_stream(args)
        return
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the serving sweep measures the GPU request loop; the CPU arm is "
                              "timed on the batch workloads"}), flush=True)
            return
        args.pairs = 1000 if args.pairs is None else args.pairs
        args.steps = 3 if args.steps is None else args.steps
        run_serve(args)
        return
    # Defaults per workload: pairs, plain per-call sample, CPU sample (about
    # 10-30 s of CPU work on a 16-core host).
    pairs, plain, cpu, steps = {"shortread": (1_000_000, 2000, 1_000_000, 40),
                                "small": (10_000, 2000, 10_000, 40),
                                "longread": (20_000, 8, 160, 3),
                                "extension": (200_000, 200, 20_000, 5)}[args.workload]
    args.steps = steps if args.steps is None else args.steps
    args.pairs = pairs if args.pairs is None else args.pairs
    args.plain_pairs = plain if args.plain_pairs is None else args.plain_pairs
    args.cpu_sample = cpu if args.cpu_sample is None else args.cpu_sample
    args.parity_pairs = cpu if args.parity_pairs is None else args.parity_pairs
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
