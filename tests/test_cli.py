"""The align_benchmark-compatible driver on CPU: input parsing, option
parsing and the option checks that end a run before anything is aligned."""
import importlib

import pytest

from _pkg import load


@pytest.fixture(scope="module")
def cli():
    load()
    return importlib.import_module("wfa_b200.align_benchmark")


def test_read_pairs(cli, tmp_path):
    f = tmp_path / "x.seq"
    f.write_bytes(b">ACGT\r\n<ACGA\r\nTTT\nTTA\n>G\n")
    assert cli.read_pairs(str(f)) == [(b"ACGT", b"ACGA"), (b"TTT", b"TTA")]


def test_parse_span_and_proportions(cli):
    assert cli.parse_span(None) == ("global", None)
    assert cli.parse_span("extend") == ("extension", None)
    assert cli.parse_span("ends-free,0,0.5,1,7") == ("ends-free", [0.0, 0.5, 1.0, 7.0])
    assert cli.nominal_prop(10, 0.5) == 5 and cli.nominal_prop(10, 7) == 7
    with pytest.raises(SystemExit):
        cli.parse_span("ends-free,1,2")
    with pytest.raises(SystemExit):
        cli.parse_span("local")


def test_parse_heuristic(cli):
    assert cli.parse_heuristic("xdrop", "200,1") == ("xdrop", [200, 1])
    assert cli.parse_heuristic("banded-static", "-5,5") == ("banded-static", [-5, 5])
    for bad in [("xdrop", "200"), ("nope", "1"), ("wfa-adaptive", "1,2")]:
        with pytest.raises(SystemExit):
            cli.parse_heuristic(*bad)


@pytest.mark.parametrize("argv", [
    ["--wfa-memory", "ultralow", "--wfa-span", "extension"],
    ["--wfa-memory", "ultralow", "--wfa-heuristic", "zdrop", "--wfa-heuristic-parameters", "10,1"],
    ["-a", "edit-wfa", "--wfa-heuristic", "xdrop", "--wfa-heuristic-parameters", "10,1"],
    ["-a", "blast"],
    ["--wfa-memory", "tiny"],
])
def test_rejected_presets(cli, tmp_path, argv):
    f = tmp_path / "x.seq"
    f.write_bytes(b">A\n<A\n")
    with pytest.raises(SystemExit) as e:
        cli.main(["-i", str(f)] + argv)
    assert e.value.code == 1
