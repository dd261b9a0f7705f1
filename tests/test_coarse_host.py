"""Host construction of the two-level preconditioner's coarse space (no GPU):
the coarse lattice sizes and the inverse of P^T Z P from the library's
Cholesky against NumPy, with Z taken from the CPU oracle on generated
cavity and duct decks.  FP64 throughout: relative 1e-10."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rel_l2


def _hats(n, s=4.0):
    if n < 2:
        return sp.csr_matrix(np.ones((n, 1)))
    cd = max(2, min(int(np.ceil((n - 1) / s - 1e-9)) + 1, n))
    h = (n - 1) / (cd - 1)
    x = np.arange(n)
    i = np.clip(np.floor(x / h).astype(int), 0, cd - 2)
    f = np.clip(x / h - i, 0.0, 1.0)
    return sp.csr_matrix((np.concatenate([1 - f, f]), (np.concatenate([x, x]), np.concatenate([i, i + 1]))),
                         shape=(n, cd))


@pytest.mark.parametrize("case", ["cavity", "duct"])
def test_coarse_inverse_matches_numpy(case, tmp_path, oracle_mod):
    import cfdfs
    from cfdfs import meshgen
    if case == "cavity":
        deck = meshgen.write_cavity(str(tmp_path / "c.inp"), meshgen.CavitySpec(12, re=100, dt=0.01, steps=2, ngp=8))
        dims = (13, 13, 13)
    else:
        deck = meshgen.write_duct(str(tmp_path / "d.inp"), n_cross=4, n_axial=24, steps=2, dt=0.01)
        dims = meshgen.duct_grid_dims(4, 24)
    o = oracle_mod.Oracle(deck)
    o.step0()
    Z = o.csr("Z").tocsr()
    o.close()
    cd, inv = cfdfs.coarse_inverse(dims, Z.indptr, Z.indices, Z.data)
    P = sp.kron(_hats(dims[2]), sp.kron(_hats(dims[1]), _hats(dims[0]))).tocsr()
    assert cd == tuple(_hats(n).shape[1] for n in dims)
    ref = np.linalg.inv((P.T @ Z @ P).toarray())
    assert rel_l2(inv, ref) < 1e-10
    assert np.allclose(inv, inv.T, rtol=0, atol=1e-12 * np.abs(inv).max())


def test_coarse_lattice_limits():
    import cfdfs
    # spacing 4 voxels where the axis allows; widened beyond 6000 nodes
    rp = np.zeros(1, dtype=np.int32)
    L = cfdfs.lib()
    import ctypes as C
    for dims, want in (((65, 65, 65), (17, 17, 17)), ((161, 25, 25), (41, 7, 7)), ((9, 9, 9), (3, 3, 3))):
        d = np.array(dims, dtype=np.int32)
        cd = np.zeros(3, dtype=np.int32)
        assert L.cfdh_coarse_inverse(cfdfs._p(d, C.c_int), cfdfs._p(rp, C.c_int), cfdfs._p(rp, C.c_int),
                                     cfdfs._p(np.zeros(1), C.c_double), cfdfs._p(cd, C.c_int), None) == 0
        assert tuple(cd) == want
    d = np.array((257, 257, 257), dtype=np.int32)
    cd = np.zeros(3, dtype=np.int32)
    L.cfdh_coarse_inverse(cfdfs._p(d, C.c_int), cfdfs._p(rp, C.c_int), cfdfs._p(rp, C.c_int),
                          cfdfs._p(np.zeros(1), C.c_double), cfdfs._p(cd, C.c_int), None)
    assert int(np.prod(cd)) <= 6000


def _laplace7(dims, shift):
    """Shifted 7-point Laplacian on an x-fastest grid: a synthetic SPD Z."""
    nx, ny, nz = dims
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.full(n, 6.0 + shift)]
    for ax in range(3):
        a = np.moveaxis(idx, 2 - ax, 0)
        lo, hi = a[:-1].ravel(), a[1:].ravel()
        rows += [lo, hi]
        cols += [hi, lo]
        vals += [np.full(lo.size, -1.0), np.full(lo.size, -1.0)]
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


@pytest.mark.parametrize("dims", [(25, 25, 25), (29, 21, 17)])
def test_coarse_inverse_multi_panel(dims):
    """Coarse sizes of 343 and 240 nodes: more than one 96-column panel of
    the blocked Cholesky, with edge tiles of the 4 x 4 register-tiled
    trailing update and of the row-tiled inverse."""
    import cfdfs
    Z = _laplace7(dims, 0.05)
    Z.sort_indices()
    cd, inv = cfdfs.coarse_inverse(dims, Z.indptr.astype(np.int32), Z.indices.astype(np.int32), Z.data)
    P = sp.kron(_hats(dims[2]), sp.kron(_hats(dims[1]), _hats(dims[0]))).tocsr()
    assert cd == tuple(_hats(n).shape[1] for n in dims)
    assert int(np.prod(cd)) > 96 * 2
    ref = np.linalg.inv((P.T @ Z @ P).toarray())
    assert rel_l2(inv, ref) < 1e-10


def _hats_s(n, s):
    return _hats(n, s)


@pytest.mark.parametrize("case,spacing", [("cavity", 4.0), ("duct", 4.0), ("cavity", 3.0)])
def test_coarse_matrix_matches_scipy(case, spacing, tmp_path, oracle_mod):
    """The Galerkin product itself (cfdh_coarse_matrix, the host build that
    the device build reproduces bit for bit) against SciPy's P^T Z P."""
    import cfdfs
    from cfdfs import meshgen
    if case == "cavity":
        deck = meshgen.write_cavity(str(tmp_path / "c.inp"), meshgen.CavitySpec(12, re=100, dt=0.01, steps=2, ngp=8))
        dims = (13, 13, 13)
    else:
        deck = meshgen.write_duct(str(tmp_path / "d.inp"), n_cross=4, n_axial=24, steps=2, dt=0.01)
        dims = meshgen.duct_grid_dims(4, 24)
    o = oracle_mod.Oracle(deck)
    o.step0()
    Z = o.csr("Z").tocsr()
    o.close()
    cd, zc = cfdfs.coarse_matrix(dims, Z.indptr, Z.indices, Z.data, spacing=spacing)
    P = sp.kron(_hats_s(dims[2], spacing), sp.kron(_hats_s(dims[1], spacing), _hats_s(dims[0], spacing))).tocsr()
    assert cd == tuple(_hats_s(n, spacing).shape[1] for n in dims)
    ref = (P.T @ Z @ P).toarray()
    assert rel_l2(zc, ref) < 1e-13
    assert np.array_equal(zc, zc.T)
