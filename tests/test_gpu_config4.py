"""The ends-free / extension workload (flanked long pairs with heuristics) on
the GPU through the C ABI against the oracle, bit-exact: the extension span
with X-drop and Z-drop 200, and the ends-free span with WF-adaptive (10, 50),
under gap-affine, edit and indel, score-only and with CIGAR."""
import pytest

from _pkg import load
from test_emu_vs_oracle import HEUR
from test_gpu_parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return load()


@pytest.fixture(scope="module")
def pairs():
    from wfa_b200 import synth
    ps = synth.config4(24, seed=0xC4)
    return [ps.pair(i) for i in range(len(ps))]


@pytest.mark.parametrize("compute", [True, False])
@pytest.mark.parametrize("h", ["xdrop", "zdrop"])
def test_extension_with_drops(pkg, pairs, h, compute):
    compare(pkg, 3, [0, 4, 6, 2], pairs, compute=compute, extension=True, hk=HEUR[h], hp=(200, 1, 0))


@pytest.mark.parametrize("compute", [True, False])
@pytest.mark.parametrize("metric,pen", [(3, [0, 4, 6, 2]), (1, None), (0, None)])
def test_endsfree_with_adaptive(pkg, pairs, metric, pen, compute):
    compare(pkg, metric, pen, pairs, compute=compute, span=1, free=(300, 300, 300, 300),
            hk=HEUR["wfa-adaptive"], hp=(10, 50, 1))
