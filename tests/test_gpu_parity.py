"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same generated decks.  Tolerances: relative L2 <= 1e-12 for assembled
operators, <= 1e-9 for single stages and solves, <= 1e-6 (FP64) for whole
runs, as the FP64 target of the solver."""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12
STAGE_TOL = 1e-9
RUN_TOL = 1e-6


def _pair(decks, oracle_mod, key, **kw):
    import cfdfs
    o = oracle_mod.Oracle(decks[key], ngp=kw.get("ngp", 0))
    o.step0()
    s = cfdfs.Solver(device=0, **kw)
    s.load(decks[key])
    s.step0()
    return o, s


@pytest.mark.parametrize("key", ["c1", "c1_27", "perturbed", "duct_small"])
def test_operators_match_oracle(decks, oracle_mod, key):
    o, s = _pair(decks, oracle_mod, key)
    rp, col, kv = s.matrix("K")
    orp, ocol = o.pattern("K")
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert rel_l2(kv, o.values("K")) < OP_TOL
    g_rp, g_col, gv = s.matrix("G")
    for d, name in enumerate(("G1", "G2", "G3")):
        assert rel_l2(gv[:, d], o.values(name)) < OP_TOL, name
    rp, col, zv = s.matrix("Z")
    orp, ocol = o.pattern("Z")
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert rel_l2(zv, o.values("Z")) < OP_TOL
    assert rel_l2(s.vector("MdOrigInv"), o.vec("MdOrigInv")) < OP_TOL
    assert rel_l2(s.vector("MdInv"), o.vec("MdInv")) < OP_TOL
    # G^T values are the transpose of G
    import scipy.sparse as sp
    rpt, colt, gtv = s.matrix("GT")
    G1 = sp.csr_matrix((gv[:, 0], g_col, g_rp), shape=(len(g_rp) - 1, o.NNp)).T.tocsr()
    G1.sort_indices()
    assert np.array_equal(G1.data, gtv[:, 0])
    s.close()
    o.close()


def test_pressure_solve_matches_oracle(decks, oracle_mod):
    o, s = _pair(decks, oracle_mod, "c1")
    rng = np.random.default_rng(3)
    b = rng.standard_normal(o.NNp)
    b[o.zero_p] = 0.0
    o.set_cg(1e-8, 1000, 0)
    xo, st_o = o.cg(b)
    xg, st_g = s.pressure_solve(b)
    assert st_g.status == 0 and st_o[2] == 0
    assert abs(st_g.iterations - st_o[0]) <= 2
    assert rel_l2(xg, xo) < 1e-7
    Z = o.csr("Z")
    assert np.linalg.norm(b - Z @ xg) <= 1.01e-8 * np.linalg.norm(b)
    s.close()
    o.close()


def _stage_compare(o, s, it, compare_norms):
    """Runs sub-iteration `it` on both from identical state and compares."""
    o.step1(it)
    s.calculateMatrixAGPU()
    s.step1GPUpart(it)
    assert rel_l2(s.vector("R1"), o.vec("R1")) < STAGE_TOL
    assert rel_l2(s.vector("UnpHalf"), o.vec("UnpHalf")) < STAGE_TOL
    st_o = o.step2(it)
    st_g = s.step2GPU(it)
    assert rel_l2(s.vector("R2"), o.vec("R2")) < STAGE_TOL
    assert rel_l2(s.vector("Pdot"), o.vec("Pdot")) < 1e-7
    assert abs(st_g.iterations - st_o[0]) <= 2
    o.step3(it)
    s.step3GPU(it)
    assert rel_l2(s.vector("Unp1"), o.vec("Unp1")) < 1e-7
    assert rel_l2(s.vector("Acc"), o.vec("Acc")) < 1e-6
    co, no = o.check_iter()
    cg, ng = s.checkConvergenceGPU()
    if compare_norms:
        assert co == cg
        assert np.allclose(no, ng, rtol=1e-5, atol=0)


def test_stages_match_oracle_from_same_state(decks, oracle_mod):
    o, s = _pair(decks, oracle_mod, "c1")
    o.run(3)                                   # develop a flow on the oracle
    s.set_state(o.vec("Un"), o.vec("Pn"))      # and hand the same state to the GPU
    o.begin_step()
    s.begin_step()
    assert rel_l2(s.vector("UnpHalf_prev"), o.vec("UnpHalf_prev")) == 0.0
    # iteration 1: Unp1_prev differs (the oracle carries the stale vector of
    # the C++ loop), so the convergence norms are compared from iteration 2
    _stage_compare(o, s, 1, compare_norms=False)
    o.rotate()
    s.rotate()
    s.calculate_KtimesAcc_prevGPU()
    assert rel_l2(s.vector("KtimesAcc_prev"), o.vec("KtimesAcc_prev")) < 1e-6
    _stage_compare(o, s, 2, compare_norms=True)
    s.close()
    o.close()


@pytest.mark.parametrize("key,steps", [("c1", 20), ("c1_27", 20), ("perturbed", 5), ("graded", 5),
                                       ("duct_small", 3)])
def test_full_run_fp64(decks, oracle_mod, key, steps):
    o, s = _pair(decks, oracle_mod, key)
    info_o = o.run(-1)
    st = s.run(-1)
    assert st.steps == info_o["steps"] == steps
    Ug, Pg = s.state()
    e_u = rel_l2(Ug, o.vec("Un"))
    e_p = rel_l2(Pg, o.vec("Pn"))
    assert e_u < RUN_TOL and e_p < RUN_TOL, (e_u, e_p)
    assert abs(st.cg_iters - info_o["cg_its"]) <= 2 * st.subiters
    assert st.subiters == info_o["subits"]
    s.close()
    o.close()


def test_exhausted_subiterations_match_oracle(decks, oracle_mod):
    """With a sub-iteration limit of 2, every step runs out of sub-iterations
    and ends with a rotation; the reference copies the vectors there, so the
    new state is the last iterate (the pointer-swapping rotation must hand
    over the same vectors)."""
    o, s = _pair(decks, oracle_mod, "c1_runout")
    info_o = o.run(-1)
    st = s.run(-1)
    assert st.steps == info_o["steps"] == 5
    assert st.subiters == info_o["subits"] == 10 and st.last_iter == 3
    Ug, Pg = s.state()
    assert rel_l2(Ug, o.vec("Un")) < RUN_TOL and rel_l2(Pg, o.vec("Pn")) < RUN_TOL
    s.close()
    o.close()


def test_stage_driver_equals_fused_run(decks, oracle_mod):
    """cfd_run and the stage-by-stage entry points give the same result."""
    import cfdfs
    a = cfdfs.Solver(device=0)
    a.load(decks["c1"])
    a.step0()
    b = cfdfs.Solver(device=0)
    b.load(decks["c1"])
    b.step0()
    a.run(4)
    for _ in range(4):
        b.time_step()
    Ua, Pa = a.state()
    Ub, Pb = b.state()
    assert rel_l2(Ua, Ub) < 1e-12 and rel_l2(Pa, Pb) < 1e-12
    a.close()
    b.close()


def test_mixed_precision_error(decks, oracle_mod):
    import cfdfs
    o, s = _pair(decks, oracle_mod, "c1", precision=cfdfs.MIXED)
    o.run(-1)
    s.run(-1)
    Ug, Pg = s.state()
    e_u = rel_l2(Ug, o.vec("Un"))
    e_p = rel_l2(Pg, o.vec("Pn"))
    # mixed precision: FP32 operators, FP64 state and refinement
    assert e_u < 1e-5 and e_p < 1e-5, (e_u, e_p)
    s.close()
    o.close()


def test_tecplot_and_restart_roundtrip(decks, oracle_mod, tmp_path):
    o, s = _pair(decks, oracle_mod, "c1")
    s.run(5)
    U, P = s.state()
    o.set_vec("Un", U)
    o.set_vec("Pn", P)
    pg, po = str(tmp_path / "g.dat"), str(tmp_path / "o.dat")
    s.write_tecplot(pg, "cavity")
    o.write_tecplot(po, "cavity")
    assert open(pg).read() == open(po).read()       # same text, byte for byte
    s2 = __import__("cfdfs").Solver(device=0)
    s2.load(decks["c1"])
    s2.read_restart(pg)
    U2, P2 = s2.state()
    assert rel_l2(U2, U) < 1e-10 and rel_l2(P2, P) < 1e-10
    s.close()
    s2.close()
    o.close()


def test_failures_are_reported_not_hung(decks):
    import cfdfs
    s = cfdfs.Solver(device=0, cg_maxit=1)
    s.load(decks["c1"])
    s.step0()
    rng = np.random.default_rng(1)
    x, st = s.pressure_solve(rng.standard_normal(s.info.NNp))
    assert st.status == 1 and st.iterations == 1          # iteration limit reported
    # a bounded device wait on a flag nothing sets returns a timeout status
    assert s.selftest_wait_timeout(50) == cfdfs.CFD_E_TIMEOUT
    # the context stays usable afterwards
    x, st = s.pressure_solve(rng.standard_normal(s.info.NNp))
    assert st.status == 1
    # non-finite input is reported
    U, P = s.state()
    U[5] = np.nan
    s.set_state(U, P)
    s.begin_step()
    s.calculateMatrixAGPU()
    s.step1GPUpart(1)
    with pytest.raises(cfdfs.CfdError) as ei:
        s.step2GPU(1)
    assert ei.value.code == cfdfs.CFD_E_NONFINITE
    s.close()


def _det_run(path, steps, weights=None, **kw):
    import cfdfs
    s = cfdfs.Solver(device=0, deterministic=1, **kw)
    s.load(path)
    s.step0()
    if weights:
        s.load_unet(weights)
    ops = [s.matrix(w)[2].copy() for w in ("K", "G", "Z")]
    st = s.run(steps)
    U, P = s.state()
    s.close()
    return ops, st, U, P


@pytest.mark.parametrize("key", ["c1", "c1_27", "perturbed"])
def test_deterministic_mode(decks, oracle_mod, key):
    """Coloured assembly and convection without atomics: the oracle's
    operators and run to the usual tolerances, and two runs in separate
    contexts bitwise identical (operators, velocity and pressure)."""
    o = oracle_mod.Oracle(decks[key])
    o.step0()
    info_o = o.run(-1)
    steps = info_o["steps"]
    ops1, st1, U1, P1 = _det_run(decks[key], steps)
    ops2, st2, U2, P2 = _det_run(decks[key], steps)
    assert rel_l2(ops1[0], o.values("K")) < OP_TOL
    assert rel_l2(ops1[2], o.values("Z")) < OP_TOL
    assert st1.steps == steps
    assert rel_l2(U1, o.vec("Un")) < RUN_TOL and rel_l2(P1, o.vec("Pn")) < RUN_TOL
    for a, b in zip(ops1, ops2):
        assert np.array_equal(a, b)
    assert np.array_equal(U1, U2) and np.array_equal(P1, P2)
    assert st1.cg_iters == st2.cg_iters
    o.close()


def test_deterministic_mixed_twolevel(decks):
    """The mixed two-level path is bitwise reproducible in deterministic mode
    (its Krylov reductions are fixed-order block sums already)."""
    import cfdfs
    kw = dict(precision=cfdfs.MIXED, precond=cfdfs.PC_TWOLEVEL)
    _, st1, U1, P1 = _det_run(decks["c1"], 6, **kw)
    _, st2, U2, P2 = _det_run(decks["c1"], 6, **kw)
    assert np.array_equal(U1, U2) and np.array_equal(P1, P2)
    assert st1.cg_iters == st2.cg_iters


def test_deterministic_mixed_learned(decks):
    """The mixed learned path (the committed network in the first iteration
    of each pressure solve, flexible CG, Jacobi-PCG fallback on a stall) is
    bitwise reproducible in deterministic mode: the same fallback decisions,
    iteration counts and fields in two runs."""
    import os
    import cfdfs
    w = os.path.join(os.path.dirname(cfdfs.__file__), "..", "weights", "unet_cavity.bin")
    kw = dict(precision=cfdfs.MIXED, precond=cfdfs.PC_LEARNED, fcg_net_iters=1)
    _, st1, U1, P1 = _det_run(decks["c1"], 8, weights=w, **kw)
    _, st2, U2, P2 = _det_run(decks["c1"], 8, weights=w, **kw)
    assert np.array_equal(U1, U2) and np.array_equal(P1, P2)
    assert st1.cg_iters == st2.cg_iters and st1.fallbacks == st2.fallbacks
