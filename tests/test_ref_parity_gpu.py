"""Parity of the GPU path with the reference itself.

The fixtures ``tests/golden/ref_<case>.npz`` hold what the reference's own
CPU solver (fractionalStep/Cpp/blascoCodinaHuerta.cpp compiled unmodified
against the stand-in MKL and CSparse of ``oracle/refshim``; see
``tests/golden/make_ref_goldens.py``) printed and wrote.  The GPU runs use
the reference's pressure solve: Jacobi-PCG from x0 = 0 to
||r||_2 <= 1e-6 ||b||_2 (MKL dcg, dpar[0] = 1e-12 on squared norms,
blascoCodinaHuerta.cpp:3998-4018).

Tolerances: relative L2 <= 1e-6 per final field (u, v, w, p) for the FP64
path, as for every FP64 run; 1e-5 for the mixed-precision learned path.
The node numbering and element map of the Tecplot output are compared bit
for bit, the sub-iteration count of every step exactly, the CG iterations
of every pressure solve within 2 of the reference's, the monitor table row
by row in the reference's format.
"""
import os
import subprocess

import numpy as np
import pytest

import ref_cases
from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 1e-5


def _mon_norm(text):
    return text.replace("-0.00000", " 0.00000")


def _deck(name, tmp):
    text = ref_cases.deck_text(name)
    fix = ref_cases.load_fixture(name, GOLDEN)
    assert ref_cases.sha256_text(text) == str(fix["deck_sha256"]), "deck generator changed"
    path = os.path.join(str(tmp), name + ".inp")
    with open(path, "w") as f:
        f.write(text)
    return path, fix


def _check_fields(fix, dat, tol):
    assert dat["zone"] == str(fix["zone"])
    assert dat["xyz_sha"] == str(fix["xyz_sha"])
    assert dat["conn_sha"] == str(fix["conn_sha"])
    d = ref_cases.compare_summary(fix, dat["uvwp"])
    for field, r in d.items():
        for k, v in r.items():
            assert v <= tol, (field, k, v)
    return d


def _monitor_rows_match(rows, fix, rel):
    """Monitor rows: step and iteration columns exactly; the printed values
    (5 decimals) equal, or apart by at most one unit of the last printed
    digit plus ``rel`` of the value (a difference within the run's
    tolerance that crosses a rounding boundary; maxAcc = max|dU|/dt
    magnifies velocity differences by 1/dt)."""
    rows = np.asarray(rows)
    assert rows.shape == fix["mon"].shape
    assert np.array_equal(rows[:, :2], fix["mon"][:, :2])
    ours = [_mon_norm(ref_cases.monitor_text(*r)) for r in rows]
    theirs = [_mon_norm(t) for t in fix["mon_text"]]
    for a, b in zip(ours, theirs):
        if a != b:
            va = np.array([float(x) for x in a.split()[2:]])
            vb = np.array([float(x) for x in b.split()[2:]])
            assert np.all(np.abs(va - vb) <= 1.01e-5 + rel * np.abs(vb)), (a, b)


@pytest.mark.parametrize("name", ref_cases.GPU_CASES)
def test_stage_loop_fp64_matches_reference(name, tmp_path):
    """The reference's time loop driven through the stage entry points
    (cfd_begin_step ... cfd_end_step, the calls of the USECUDA seam)."""
    import cfdfs
    path, fix = _deck(name, tmp_path)
    s = cfdfs.Solver(device=0, cg_rtol=ref_cases.REF_CG_RTOL, cg_maxit=ref_cases.REF_CG_MAXIT, cg_warm=0)
    s.load(path)
    s.step0()
    rows, cg = [], []
    while True:
        i = s.refresh()
        if not (i.timeT < i.t_final):
            break
        r = s.time_step()
        i = s.refresh()
        m = s.monitor()
        rows.append([i.timeN, r["iter"], i.timeT, m[0], m[1], m[2], m[3], r["max_acc"]])
        cg += r["cg"]
        if r["steady"]:
            break
    dat_path = str(tmp_path / (name + ".dat"))
    s.write_tecplot(dat_path, name)
    s.close()
    dat = ref_cases.parse_dat(open(dat_path).read())
    _check_fields(fix, dat, FP64_TOL)
    cg = np.array(cg)
    assert cg.shape == fix["cg_iters"].shape
    assert np.max(np.abs(cg - fix["cg_iters"])) <= 2, (cg, fix["cg_iters"])
    _monitor_rows_match(rows, fix, 2e-6)


@pytest.mark.parametrize("name", ["c1", "steady", "c16"])
def test_fused_run_fp64_matches_reference(name, tmp_path):
    """cfd_run (the whole loop on the device) against the reference: final
    fields, step count, sub-iterations and the steady-state stop."""
    import cfdfs
    path, fix = _deck(name, tmp_path)
    s = cfdfs.Solver(device=0, cg_rtol=ref_cases.REF_CG_RTOL, cg_maxit=ref_cases.REF_CG_MAXIT, cg_warm=0)
    s.load(path)
    s.step0()
    max_iter = s.refresh().maxIter
    st = s.run(-1)
    dat_path = str(tmp_path / (name + ".dat"))
    s.write_tecplot(dat_path, name)
    s.close()
    mon = fix["mon"]
    assert st.steps == len(mon)
    # the monitor's Iter column is maxIter + 1 for a step whose loop ran out
    assert st.subiters == int(np.minimum(mon[:, 1], max_iter).sum())
    assert bool(st.steady) == (name == "steady")
    assert abs(st.maxAcc - mon[-1, 7]) <= 1e-5 * max(1.0, abs(mon[-1, 7]))
    _check_fields(fix, ref_cases.parse_dat(open(dat_path).read()), FP64_TOL)


def _fs_solver(tmp_path, name, env):
    exe = os.path.join(ROOT, "cfd-with-cuda_b200", "bin", "fs_solver")
    with open(tmp_path / "ProblemName.txt", "w") as f:
        f.write(name + "\n")
    p = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, CFD_DEVICE="0", **env))
    assert p.returncode == 0, p.stderr[-2000:]
    return p.stdout


@pytest.mark.parametrize("name", ["c1", "steady"])
def test_fs_solver_fp64_matches_reference(name, tmp_path):
    """The command-line driver with the reference's contract: ProblemName.txt
    -> <name>.inp -> <name>.dat and the monitor table on stdout."""
    _, fix = _deck(name, tmp_path)
    out = _fs_solver(tmp_path, name, {"CFD_CG_RTOL": repr(ref_cases.REF_CG_RTOL)})
    _, mon, _ = ref_cases.parse_stdout(out)
    assert "Time step  Iter     Time       u_monitor" in out
    _monitor_rows_match(mon, fix, 2e-6)
    _check_fields(fix, ref_cases.parse_dat(open(tmp_path / (name + ".dat")).read()), FP64_TOL)


def test_fs_solver_mixed_learned_matches_reference(tmp_path):
    """fs_solver with the mixed-precision learned preconditioner (the
    committed network) on the 8^3 cavity, within the mixed bound."""
    name = "c1"
    _, fix = _deck(name, tmp_path)
    out = _fs_solver(tmp_path, name, {"CFD_CG_RTOL": repr(ref_cases.REF_CG_RTOL), "CFD_PRECISION": "mixed",
                                      "CFD_PRECOND": "learned"})
    _, mon, _ = ref_cases.parse_stdout(out)
    assert mon.shape == fix["mon"].shape
    assert np.array_equal(mon[:, :2], fix["mon"][:, :2])
    _check_fields(fix, ref_cases.parse_dat(open(tmp_path / (name + ".dat")).read()), MIXED_TOL)
