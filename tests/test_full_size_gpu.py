"""Whole runs at full configuration size against golden end states of the
FP64 CPU oracle (made by tests/golden/make_run_goldens.py, which runs the
oracle for minutes; too long to repeat on every test run):

- the 32^3 cavity at Re 400, 200 steps (the FP64 drop-in configuration), by
  the FP64 Jacobi-PCG path and by the mixed-precision learned path;
- the 64^3 cavity at Re 1000, dt 0.002, 100 steps (the configuration of the
  headline benchmark), by the same two paths;
- the bent square duct, 24 x 24 x 160 elements, Re 200, 300 steps, parabolic
  inlet, by the same two paths.

A golden file holds a strided subsample of the final velocity and pressure,
the norms of the whole fields and the run counters.  Tolerances (relative L2
on the subsample and relative difference of the norms): 1e-6 for FP64 runs,
as the FP64 parity bound of whole runs, and 1e-5 for mixed runs, the
per-field bound of the mixed solver against FP64."""
import importlib.util
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(os.path.dirname(HERE), "cfd-with-cuda_b200", "weights", "unet_cavity.bin")
FP64_TOL = 1e-6
MIXED_TOL = 1e-5


def _cases():
    spec = importlib.util.spec_from_file_location("make_run_goldens",
                                                  os.path.join(HERE, "golden", "make_run_goldens.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _dims(case):
    from cfdfs import meshgen
    c = _cases().CASES[case]
    if c["kind"] == "duct":
        return meshgen.duct_grid_dims(c["n_cross"], c["n_axial"])
    return (c["n"] + 1,) * 3


def _run(case, tmp_path, precision, learned):
    import cfdfs
    g = _cases()
    deck = g.deck_for(case, str(tmp_path))
    kw = dict(precision=precision)
    if learned:
        kw.update(precond=cfdfs.PC_LEARNED, fcg_net_iters=1)
    s = cfdfs.Solver(device=0, **kw)
    s.load(deck)
    s.step0()
    dims = _dims(case)
    if learned:
        s.set_pressure_grid(dims)
        s.load_unet(WEIGHTS, dims)
    hm = cfdfs.HostMesh(deck)
    inlet = g.inlet_for(case, hm)
    hm.close()
    if inlet is not None:
        s.set_bc_values(*inlet)
    st = s.run(-1)
    U, P = s.state()
    s.close()
    return st, U, P


def _check(case, st, U, P, tol, counters):
    gd = np.load(os.path.join(HERE, "golden", f"{case}.npz"))
    assert st.steps == int(gd["steps"])
    e_u = rel_l2(U[::int(gd["u_stride"])], gd["u_sub"])
    e_p = rel_l2(P[::int(gd["p_stride"])], gd["p_sub"])
    n_u = abs(np.linalg.norm(U) / float(gd["u_norm"]) - 1.0)
    n_p = abs(np.linalg.norm(P) / float(gd["p_norm"]) - 1.0)
    assert max(e_u, e_p, n_u, n_p) < tol, (e_u, e_p, n_u, n_p)
    if counters:
        # same sub-iterations; CG iterations within 2 per solve
        assert st.subiters == int(gd["subits"])
        assert abs(st.cg_iters - int(gd["cg_its"])) <= 2 * st.subiters


@pytest.mark.parametrize("case", ["c2_cavity32", "c3_cavity64", "duct_24x160"])
def test_full_size_fp64_run_matches_oracle(case, tmp_path):
    st, U, P = _run(case, tmp_path, 0, learned=False)
    _check(case, st, U, P, FP64_TOL, counters=True)


@pytest.mark.parametrize("case", ["c2_cavity32", "c3_cavity64", "duct_24x160"])
def test_full_size_mixed_learned_run_matches_oracle(case, tmp_path):
    import cfdfs
    st, U, P = _run(case, tmp_path, cfdfs.MIXED, learned=True)
    _check(case, st, U, P, MIXED_TOL, counters=False)
