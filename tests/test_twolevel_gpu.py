"""Two-level pressure preconditioner on the GPU: Jacobi step plus the
Galerkin coarse-space correction P Zc^-1 P^T (Zc = P^T Z P on a coarse
lattice of trilinear hats over the structured pressure grid).

The device result of the preconditioner is checked against an independent
NumPy/SciPy construction of the same operator from the downloaded Z: the
device stores the coarse inverse in FP16 (scaled) and forms the coarse
product in FP32, so the bound is 1e-5 against the same rounded operator and
2e-3 against the exact one; solves reach the requested residual, agree with
Jacobi-PCG and take fewer iterations; whole runs keep the run tolerances of
the parity tests against the CPU oracle (1e-6 FP64, 1e-5 mixed)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _lattice(n, s=4.0):
    """Coarse nodes and spacing along an axis of n voxels (spacing 4)."""
    if n < 2:
        return 1, 1.0
    cd = int(np.ceil((n - 1) / s - 1e-9)) + 1
    cd = max(2, min(cd, n))
    return cd, (n - 1) / (cd - 1)


def _hats(n):
    cd, h = _lattice(n)
    x = np.arange(n)
    if cd < 2:
        return sp.csr_matrix(np.ones((n, 1))), 1
    i = np.clip(np.floor(x / h).astype(int), 0, cd - 2)
    f = np.clip(x / h - i, 0.0, 1.0)
    P = sp.csr_matrix((np.concatenate([1 - f, f]), (np.concatenate([x, x]), np.concatenate([i, i + 1]))),
                      shape=(n, cd))
    return P, cd


def _reference_precond(s, dims, r, fp16=True):
    """D^-1 r + P Zc^-1 P^T r (Zc = P^T Z P) with identity voxel numbering;
    with fp16, Zc^-1 rounded as the device stores it (scaled so that its
    largest entry is 16384, then FP16)."""
    rp, col, val = s.matrix("Z")
    n = len(rp) - 1
    Z = sp.csr_matrix((val, col, rp), shape=(n, n))
    Px, _ = _hats(dims[0])
    Py, _ = _hats(dims[1])
    Pz, _ = _hats(dims[2])
    P = sp.kron(Pz, sp.kron(Py, Px)).tocsr()  # voxel x + nx (y + ny z)
    Zi = np.linalg.inv((P.T @ Z @ P).toarray())
    if fp16:
        scale = 16384.0 / np.abs(Zi).max()
        Zi = (Zi * scale).astype(np.float16).astype(np.float64) / scale
    return r / Z.diagonal() + P @ (Zi @ (P.T @ r))


def _solver(deck, **kw):
    import cfdfs
    s = cfdfs.Solver(device=0, **kw)
    s.load(deck)
    s.step0()
    return s


@pytest.fixture(scope="module")
def cavity16(tmp_path_factory):
    from cfdfs import meshgen
    d = tmp_path_factory.mktemp("tl")
    return meshgen.write_cavity(str(d / "c16.inp"), meshgen.CavitySpec(16, re=400, dt=0.005, steps=5, ngp=8))


@pytest.mark.parametrize("case", ["cavity16", "duct"])
def test_precond_matches_scipy(case, cavity16, decks):
    import cfdfs
    from cfdfs import meshgen
    if case == "cavity16":
        deck, dims = cavity16, (17, 17, 17)
    else:
        deck, dims = decks["duct_small"], meshgen.duct_grid_dims(3, 16)
    s = _solver(deck, precond=cfdfs.PC_TWOLEVEL)
    if case == "duct":
        s.set_pressure_grid(dims)
    r = np.random.default_rng(4).standard_normal(s.refresh().NNp)
    z = s.precond_apply(r)
    # same operator (FP16 inverse): FP32 products of the coarse solve
    assert rel_l2(z, _reference_precond(s, dims, r)) < 1e-5
    # and close to the exact two-level operator
    assert rel_l2(z, _reference_precond(s, dims, r, fp16=False)) < 2e-3
    # Jacobi: the linear part is D^-1 r
    s.set_options(precond=cfdfs.PC_JACOBI)
    rp, col, val = s.matrix("Z")
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    assert rel_l2(s.precond_apply(r), r / val[col == rows]) < 1e-14
    s.close()


def test_grid_must_match(decks):
    import cfdfs
    s = _solver(decks["duct_small"], precond=cfdfs.PC_TWOLEVEL)
    with pytest.raises(cfdfs.CfdError):
        s.set_pressure_grid((17, 4, 5))
    r = np.ones(s.refresh().NNp)
    with pytest.raises(cfdfs.CfdError):  # not a cube: the grid must be declared
        s.precond_apply(r)
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_twolevel_solves_to_tolerance(cavity16, precision):
    """Random and solver-generated right-hand sides: the requested residual,
    the Jacobi-PCG solution, and fewer iterations (the gap grows with the
    grid: about 5x fewer on the 65^3 pressure grid)."""
    import cfdfs
    s_j = _solver(cavity16, precision=precision, cg_rtol=1e-10)
    s_t = _solver(cavity16, precision=precision, cg_rtol=1e-10, precond=cfdfs.PC_TWOLEVEL)
    b = np.random.default_rng(3).standard_normal(s_t.refresh().NNp)
    b[s_t.info.zeroPressureNode] = 0.0
    s_j.run(2)
    r2 = s_j.vector("R2")
    for rhs, factor in ((b, 1.0), (r2, 1.0)):
        xj, st_j = s_j.pressure_solve(rhs)
        xt, st_t = s_t.pressure_solve(rhs)
        assert st_j.status == 0 and st_t.status == 0 and st_t.fallback == 0
        _, nr = s_j.pressure_residual(rhs, xt)
        assert nr <= 1.01e-10 * np.linalg.norm(rhs)
        assert rel_l2(xt, xj) < 1e-6
        assert st_t.iterations < factor * st_j.iterations, (st_t.iterations, st_j.iterations)
    s_j.close()
    s_t.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_twolevel_run_matches_oracle(decks, oracle_mod, precision):
    import cfdfs
    o = oracle_mod.Oracle(decks["c1"])
    o.step0()
    o.run(-1)
    s = _solver(decks["c1"], precision=precision, precond=cfdfs.PC_TWOLEVEL)
    st = s.run(-1)
    assert st.steps == 20 and st.fallbacks == 0
    Ug, Pg = s.state()
    tol = 1e-6 if precision == 0 else 1e-5
    assert rel_l2(Ug, o.vec("Un")) < tol and rel_l2(Pg, o.vec("Pn")) < tol
    s.close()
    o.close()


def test_split_iteration_matches_sequential(cavity16, monkeypatch):
    """The FP32 two-level iteration with the coarse solve beside the SpMV
    (w = Z D^-1 r + (Z P) e) against the sequential form (w = Z z): the same
    tolerance in about the same iterations and the same solution and run to
    FP32 rounding; the bits differ, which shows the split form ran (every
    kernel of both forms is deterministic)."""
    import cfdfs
    kw = dict(precision=cfdfs.MIXED, precond=cfdfs.PC_TWOLEVEL, cg_rtol=1e-10)
    monkeypatch.setenv("CFD_FCG_SPLIT", "0")
    s_seq = _solver(cavity16, **kw)
    monkeypatch.setenv("CFD_FCG_SPLIT", "1")
    s_spl = _solver(cavity16, **kw)
    b = np.random.default_rng(5).standard_normal(s_spl.refresh().NNp)
    b[s_spl.info.zeroPressureNode] = 0.0
    x1, st1 = s_seq.pressure_solve(b)
    x2, st2 = s_spl.pressure_solve(b)
    assert st1.status == 0 and st2.status == 0 and st2.fallback == 0
    assert abs(st1.iterations - st2.iterations) <= 2, (st1.iterations, st2.iterations)
    _, nr = s_spl.pressure_residual(b, x2)
    assert nr <= 1.01e-10 * np.linalg.norm(b)
    assert rel_l2(x2, x1) < 1e-7
    assert not np.array_equal(x1, x2)
    s_seq.run(4)
    s_spl.run(4)
    U1, P1 = s_seq.state()
    U2, P2 = s_spl.state()
    assert rel_l2(U2, U1) < 1e-7 and rel_l2(P2, P1) < 1e-6
    s_seq.close()
    s_spl.close()
