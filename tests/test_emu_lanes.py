"""The device aligner with a full 32-lane warp, or an 8-lane group (the
short-pair kernel's), emulated by host threads.

Lane partitioning of the diagonals, the warp reductions behind trims,
termination and heuristics, and warp-uniform control flow (a lane that
diverges at a barrier would hang or abort) are exercised here on CPU.
Kept small: every emulated pair costs 32 host threads.
"""
import pytest

import emu_lib
from test_emu_vs_oracle import HEUR, oracle_run
from test_oracle_unit import lcg_pairs

CASES = [
    (3, [0, 4, 6, 2], 0, None, 0, (0, 0, 0)),
    (4, [0, 4, 6, 2, 24, 1], 0, None, 0, (0, 0, 0)),
    (1, None, 0, None, 0, (0, 0, 0)),
    (2, [-1, 3, 2], 1, [6, 6, 6, 6], 0, (0, 0, 0)),
    (3, [-3, 5, 3, 2], 1, [4, 9, 4, 9], 0, (0, 0, 0)),
    (3, [0, 4, 6, 2], 0, None, HEUR["wfa-adaptive"], (10, 50, 1)),
    (3, [0, 4, 6, 2], 0, None, HEUR["xdrop"], (20, 1, 0)),
    (3, [0, 4, 6, 2], 0, None, HEUR["zdrop"], (20, 1, 0)),
    (4, [0, 4, 6, 2, 24, 1], 0, None, HEUR["banded-adaptive"], (-3, 3, 1)),
    (0, None, 0, None, HEUR["banded-static"], (-5, 5, 0)),
]


@pytest.mark.parametrize("lanes", [32, 8])
@pytest.mark.parametrize("metric,pen,span,free,hk,hp", CASES)
def test_lane_groups(metric, pen, span, free, hk, hp, lanes):
    pairs = lcg_pairs(101 + metric + hk, 3, 260)
    res, cig = emu_lib.run(metric, pen, pairs, span=span, free=free, heuristic=hk, hparams=hp,
                           lanes=lanes, packed=metric == 3)
    for i, (p, t) in enumerate(pairs):
        s, st, ops, ep, _ = oracle_run(metric, pen, p, t, True, span, free, hk, list(hp))
        assert (int(res["score"][i]), int(res["status"][i]), cig[i]) == (s, st, ops), i


# Med/low (the piggyback backtrace) and Compat::Corrected ends-free with a
# match reward (candidate, diagonal pruning, begin-free dominance pruning).
CASES_MODES = [
    (3, [0, 4, 6, 2], 0, None, "med", 0),
    (4, [0, 4, 6, 2, 24, 1], 1, [5, 5, 5, 5], "low", 0),
    (2, [-1, 3, 2], 1, [3, 12, 3, 12], "high", 1),
    (3, [-3, 5, 3, 2], 1, [2, 40, 2, 40], "med", 1),
    (4, [-1, 4, 6, 2, 24, 1], 1, [260, 260, 260, 260], "high", 1),
]


@pytest.mark.parametrize("metric,pen,span,free,memory,compat", CASES_MODES)
def test_32_lanes_memory_modes_and_corrected(metric, pen, span, free, memory, compat):
    pairs = lcg_pairs(131 + metric, 3, 200)
    fr = None
    if free:
        fr = [min(free[0], min(len(p) for p, _ in pairs)), min(free[1], min(len(p) for p, _ in pairs)),
              min(free[2], min(len(t) for _, t in pairs)), min(free[3], min(len(t) for _, t in pairs))]
    res, cig = emu_lib.run(metric, pen, pairs, span=span, free=fr, lanes=32,
                           piggyback=memory if memory != "high" else False, compat=compat)
    for i, (p, t) in enumerate(pairs):
        s, st, ops, ep, _ = oracle_run(metric, pen, p, t, True, span, fr, 0, [0, 0, 0],
                                       memory=memory, compat=compat)
        assert (int(res["score"][i]), int(res["status"][i]), cig[i]) == (s, st, ops), i
