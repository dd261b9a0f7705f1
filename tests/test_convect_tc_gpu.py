"""Tensor-core convection (CFD_CONVECT_TC=1, mixed precision): the two
per-element contractions of the convection term (gathered nodal values x the
Gauss-point basis table, and the weighted convective products x the shape
functions) run as tcgen05 MMAs with TF32 operands split into hi + lo parts.

From the same state, step 1's R1 (convection + diffusion + pressure terms)
and the intermediate velocity agree with the CUDA-core FP32 kernel and with
the FP64 oracle to the mixed-precision stage tolerance below, on an affine
cavity, a graded cavity, a perturbed (non-affine) box whose element count
leaves a partial tile, and the bent duct; a whole mixed run agrees with the
oracle as the CUDA-core path does (test_mixed_precision_error)."""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

# FP32 operators and FP32 copies of the state in the stage: about 1e-7
# relative against FP64; the split TF32 products add about 2^-21
MIXED_STAGE_TOL = 2e-6


def _solver(deck, tc):
    import cfdfs
    os.environ["CFD_CONVECT_TC"] = "1" if tc else "0"
    try:
        s = cfdfs.Solver(device=0, precision=cfdfs.MIXED)
    finally:
        del os.environ["CFD_CONVECT_TC"]
    s.load(deck)
    s.step0()
    return s


@pytest.mark.parametrize("key", ["c1", "graded", "perturbed", "duct_small"])
def test_tc_convection_stage_matches(decks, oracle_mod, key):
    o = oracle_mod.Oracle(decks[key])
    o.step0()
    o.run(3)  # a developed flow, handed to both GPU solvers
    a, b = _solver(decks[key], True), _solver(decks[key], False)
    for s in (a, b):
        s.set_state(o.vec("Un"), o.vec("Pn"))
        s.begin_step()
        s.calculateMatrixAGPU()
        s.step1GPUpart(1)
    o.begin_step()
    o.step1(1)
    r_tc, r_cc, r_o = a.vector("R1"), b.vector("R1"), o.vec("R1")
    # the tensor-core kernel ran: its sums are rounded differently
    assert not np.array_equal(r_tc, r_cc)
    assert rel_l2(r_tc, r_cc) < MIXED_STAGE_TOL, rel_l2(r_tc, r_cc)
    assert rel_l2(r_tc, r_o) < MIXED_STAGE_TOL, (rel_l2(r_tc, r_o), rel_l2(r_cc, r_o))
    assert rel_l2(a.vector("UnpHalf"), o.vec("UnpHalf")) < MIXED_STAGE_TOL
    a.close()
    b.close()
    o.close()


def test_tc_convection_mixed_run_matches_oracle(decks, oracle_mod):
    o = oracle_mod.Oracle(decks["c1"])
    o.step0()
    s = _solver(decks["c1"], True)
    info = o.run(-1)
    st = s.run(-1)
    assert st.steps == info["steps"] == 20
    Ug, Pg = s.state()
    e_u, e_p = rel_l2(Ug, o.vec("Un")), rel_l2(Pg, o.vec("Pn"))
    assert e_u < 1e-5 and e_p < 1e-5, (e_u, e_p)
    s.close()
    o.close()


def test_tc_convection_many_tiles_per_block(tmp_path):
    """A 24^3 cavity has 864 tiles of 16 elements, more than the blocks the
    kernel launches (three per SM), so blocks run several tiles in turn and
    reuse their barriers, accumulators and shared memory: from the same
    developed state, R1 and UnpHalf agree with the CUDA-core kernel."""
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c24.inp"), meshgen.CavitySpec(24, re=400, dt=0.005, steps=5, ngp=8))
    ref = _solver(deck, False)
    ref.run(3)
    U, P = ref.state()
    ref.close()
    a, b = _solver(deck, True), _solver(deck, False)
    for s in (a, b):
        s.set_state(U, P)
        s.begin_step()
        s.calculateMatrixAGPU()
        s.step1GPUpart(1)
    r_tc, r_cc = a.vector("R1"), b.vector("R1")
    assert not np.array_equal(r_tc, r_cc)
    assert rel_l2(r_tc, r_cc) < MIXED_STAGE_TOL, rel_l2(r_tc, r_cc)
    assert rel_l2(a.vector("UnpHalf"), b.vector("UnpHalf")) < MIXED_STAGE_TOL
    a.close()
    b.close()

