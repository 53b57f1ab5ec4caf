"""The package's align_benchmark output-line module, for the tests."""
import importlib

from _pkg import load

load()
_m = importlib.import_module("wfa_b200.cli_format")
line = _m.line
rle = _m.rle
classic_score = _m.classic_score
