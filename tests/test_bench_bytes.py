"""The algorithmic byte counts behind the bench's roofline figures, on the
sizes of the 64^3 cavity (nnz from the structured-mesh formulas of
tests/golden/sizes.json): one CG SpMV pass over Z moves 0.395 GB in FP64 and
0.263 GB in FP32, one K pass over [u v w] 1.73 GB in FP64, and a time step is
the sum of its stages with the run's own iteration counts."""
import os
import sys
from types import SimpleNamespace

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

C3 = SimpleNamespace(NE=262144, NN=2146689, NNp=274625, nnzK=135005697, nnzG=33076161, nnzZ=32461759)


def test_per_pass_bytes():
    bz64 = C3.nnzZ * 12 + 4 * (C3.NNp + 1) + 2 * C3.NNp * 8
    bz32 = C3.nnzZ * 8 + 4 * (C3.NNp + 1) + 2 * C3.NNp * 4
    assert round(bz64 / 1e9, 3) == 0.395 and round(bz32 / 1e9, 3) == 0.263
    assert bench.cg_iteration_bytes(C3, False) == bz64 + 9 * C3.NNp * 8
    assert bench.cg_iteration_bytes(C3, True) == bz32 + 9 * C3.NNp * 4
    assert round(bench.algorithmic_bytes(C3, "spmv_k3", 0, False) / 1e9, 2) == 1.73


@pytest.mark.parametrize("mixed", [False, True])
def test_step_bytes_is_the_sum_of_its_stages(mixed):
    steps, subiters, cg = 20, 54, 1500
    per_sub = sum(bench.algorithmic_bytes(C3, k, 0, mixed) for k in ("convect", "step1", "gt", "step3"))
    per_sub += 12 * 3 * C3.NN * 8
    expect = (subiters * per_sub + cg * bench.cg_iteration_bytes(C3, mixed)
              + (subiters - steps) * bench.algorithmic_bytes(C3, "spmv_k3", 0, mixed)) / steps
    assert bench.step_bytes(C3, steps, subiters, cg, mixed) == pytest.approx(expect, rel=1e-15)
    assert bench.step_bytes(C3, steps, subiters, cg, mixed) > 0
