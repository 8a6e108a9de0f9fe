"""The FP64 3-D P3 flux-tile padding of the TMA element kernel
(stage_tma.cu, Tm::PADR / Tm::PADP) is the padding the shared-memory bank
model finds best for both FP64 tile shapes (2 and 4 elements per CTA)."""
import os
import re

import bank_model
from conftest import ROOT


def kernel_padding():
    src = open(os.path.join(ROOT, "flurrypp_b200", "csrc", "kernels", "stage_tma.cu")).read()
    m = re.search(r"PADR = PADDED \? (\d+) : 0, PADP = PADDED \? (\d+) : 0", src)
    assert m, "padding constants not found"
    return int(m.group(1)), int(m.group(2))


def test_padding_is_the_model_optimum():
    row, plane = kernel_padding()
    for eb in (2, 4):
        best = bank_model.best_padding(3, 8, eb, rows=range(5), planes=range(5))[0]
        chosen = bank_model.count(3, 8, eb, row, plane)
        unpadded = bank_model.count(3, 8, eb, 0, 0)
        assert chosen["sum"] == best
        assert chosen["sum"] <= 0.65 * unpadded["sum"]
        # the flux-point phases come within a sixth of the conflict-free cost
        # (2 wavefronts per 8-byte warp access of 32 distinct values, N * nF
        # accesses per warp); unpadded they cost twice that
        ideal = (6 * 16 * eb // 32) * 4 * 5 * 2
        assert chosen["C2"] == chosen["E"] <= 7 * ideal // 6
        assert unpadded["C2"] >= 2 * ideal


def test_model_counts():
    # a conflict-free warp load of 32 distinct doubles costs 2, a broadcast 1
    assert bank_model.wavefronts([8 * i for i in range(32)], 8) == 2
    assert bank_model.wavefronts([0] * 32, 8) == 1
    # 32 doubles 128 bytes apart all sit on banks 0-1
    assert bank_model.wavefronts([128 * i for i in range(32)], 8) == 32
