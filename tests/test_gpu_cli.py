"""The align_benchmark-compatible driver on the GPU against the reference's
own expected outputs (the golden cases read from its tests): the same
`score<TAB>CIGAR` lines, byte for byte, in every memory mode."""
import importlib

import pytest

from _pkg import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cli():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    load()
    return importlib.import_module("wfa_b200.align_benchmark")


def argv_for(case, seq, out):
    argv = ["-i", str(seq), "-o", str(out), "-a", case["algo"]]
    if case["penalties"]:
        opt = {"gap-linear-wfa": "--linear-penalties", "gap-affine-wfa": "--affine-penalties",
               "gap-affine2p-wfa": "--affine2p-penalties"}
        argv.append(f"{opt[case['algo']]}={case['penalties']}")  # values may start with '-'
    if case["score_only"]:
        argv.append("--wfa-score-only")
    argv += ["--wfa-memory", case["memory"], "--wfa-span", case["span"]]
    if case.get("no_c_compat"):
        argv.append("--no-c-compat")
    if case["heuristic"]:
        argv += ["--wfa-heuristic", case["heuristic"], f"--wfa-heuristic-parameters={case['hparams']}"]
    return argv


def test_golden_cases_through_the_driver(cli, golden, tmp_path):
    ran = 0
    for case in golden["cases"]:
        seq, out = tmp_path / f"{case['name']}.seq", tmp_path / f"{case['name']}.alg"
        seq.write_text("".join(f">{p}\n<{t}\n" for p, t in case["pairs"]))
        argv = argv_for(case, seq, out)
        assert cli.main(argv) == 0, case["name"]
        assert out.read_text().splitlines() == case["expected"], case["name"]
        ran += 1
    assert ran == len(golden["cases"])
