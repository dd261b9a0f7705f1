"""The persistent two-level iteration (one cooperative launch per FP32 inner
solve, csrc/cuda/fcg_persist.cu) against the per-kernel iteration replayed
from CUDA graphs (CFD_FCG_PERSIST=0): the same solves to the same
tolerances, the same step results within the mixed-precision bound, and
proof from the launch profile that each path ran."""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5


def _run(deck, precond, persist, steps, weights=None):
    import cfdfs
    os.environ["CFD_FCG_PERSIST"] = "1" if persist else "0"
    try:
        s = cfdfs.Solver(device=0, precision=cfdfs.MIXED, precond=precond,
                         fcg_net_iters=1 if precond == cfdfs.PC_LEARNED else 0)
    finally:
        del os.environ["CFD_FCG_PERSIST"]
    s.load(deck)
    s.step0()
    if weights:
        s.load_unet(weights)
    s.profile(True)
    st = s.run(steps)
    prof = s.profile_read()
    phases = s.profile_fcg2l()
    s.profile(False)
    U, P = s.state()
    s.close()
    return st, prof, phases, U, P


@pytest.mark.parametrize("kind", ["twolevel", "learned"])
def test_persistent_iteration_matches_graph_path(kind, tmp_path):
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c16.inp"), meshgen.CavitySpec(16, re=400, dt=0.005, steps=6))
    precond = cfdfs.PC_LEARNED if kind == "learned" else cfdfs.PC_TWOLEVEL
    w = os.path.join(os.path.dirname(cfdfs.__file__), "..", "weights", "unet_cavity.bin") if kind == "learned" else None
    a = _run(deck, precond, True, 6, w)
    b = _run(deck, precond, False, 6, w)
    st_a, prof_a, phases_a, Ua, Pa = a
    st_b, prof_b, _, Ub, Pb = b
    # the persistent kernel ran in one path only, and the per-kernel SpMV in the other
    assert prof_a["fcg2l"]["launches"] > 0 and prof_a["fcg2l"]["iters"] > 0
    assert prof_b["fcg2l"]["launches"] == 0 and prof_b["spmv_z"]["launches"] > 0
    assert sum(phases_a.values()) > 0
    assert st_a.steps == st_b.steps == 6 and st_a.subiters == st_b.subiters
    assert st_a.fallbacks == st_b.fallbacks == 0
    # FP32 rounding differs (coarse products summed in another order): the
    # iteration counts agree within a few per step
    assert abs(st_a.cg_iters - st_b.cg_iters) <= 2 * st_a.subiters, (st_a.cg_iters, st_b.cg_iters)
    assert rel_l2(Ua, Ub) < MIXED_TOL and rel_l2(Pa, Pb) < MIXED_TOL


def test_persistent_iteration_on_the_duct(tmp_path):
    """A non-cubic structured pressure grid (49 x 9 x 9 voxels of a small
    bent duct, axial index fastest) through the persistent iteration."""
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_duct(str(tmp_path / "duct.inp"), n_cross=8, n_axial=48, steps=3, dt=0.005)
    dims = meshgen.duct_grid_dims(8, 48)
    out = []
    for persist in (True, False):
        os.environ["CFD_FCG_PERSIST"] = "1" if persist else "0"
        try:
            s = cfdfs.Solver(device=0, precision=cfdfs.MIXED, precond=cfdfs.PC_TWOLEVEL)
        finally:
            del os.environ["CFD_FCG_PERSIST"]
        s.load(deck)
        s.step0()
        s.set_pressure_grid(dims)
        s.profile(True)
        st = s.run(3)
        prof = s.profile_read()
        s.profile(False)
        out.append((st, prof, *s.state()))
        s.close()
    (sa, pa, Ua, Pa), (sb, pb, Ub, Pb) = out
    assert pa["fcg2l"]["launches"] > 0 and pb["fcg2l"]["launches"] == 0
    assert sa.subiters == sb.subiters
    assert rel_l2(Ua, Ub) < MIXED_TOL and rel_l2(Pa, Pb) < MIXED_TOL
