"""The C-ABI library on CPU: it loads, exports every declared entry point, and
its host-only paths behave (no GPU calls here)."""
import ctypes
import os
import re

import pytest

from _pkg import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "wfa_b200.h")).read()
    return sorted(set(re.findall(r"WFA_API[^;(]*?\b(wfa_\w+)\s*\(", src, re.S)))


def test_library_exports_every_declared_symbol():
    pkg = load()
    L = pkg.lib()
    names = declared()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name


def test_penalties_check_matches_reference_validation():
    """src/penalties.rs:157-296: match <= 0; X > 0; O >= 0; E > 0."""
    pkg = load()
    from wfa_b200.aligner import Penalties
    L = pkg.lib()
    ok = lambda m, p: L.wfa_penalties_check(m, ctypes.byref(Penalties(*(p + [0] * 6)[:6])))
    assert ok(3, [0, 4, 6, 2]) == 0
    assert ok(3, [1, 4, 6, 2]) == -1
    assert ok(3, [0, 0, 6, 2]) == -1
    assert ok(3, [0, 4, -1, 2]) == -1
    assert ok(3, [0, 4, 0, 2]) == 0
    assert ok(3, [0, 4, 6, 0]) == -1
    assert ok(2, [0, 4, 2]) == 0
    assert ok(2, [0, 4, 0]) == -1
    assert ok(4, [0, 4, 6, 2, 24, 1]) == 0
    assert ok(4, [0, 4, 6, 2, 24, 0]) == -1
    assert ok(4, [-1, 4, 6, 2, 24, 1]) == 0
    assert ok(0, []) == 0 and ok(1, []) == 0


def test_rle_helper():
    pkg = load()
    assert pkg.cigar_rle(b"MMMXMMMM") == "3M1X4M"
    assert pkg.cigar_rle(b"") == ""


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pkg = load()
    with pytest.raises(RuntimeError):
        pkg.WavefrontAligner(pkg.GAP_AFFINE, [0, 4, 6, 2])
    with pytest.raises(ValueError):
        pkg.WavefrontAligner(pkg.GAP_AFFINE, [1, 4, 6, 2])
