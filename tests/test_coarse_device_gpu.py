"""The coarse-space factorisation on the device (dense_chol.cu: blocked FP64
Cholesky, forward substitution with the identity, Y^T Y) against NumPy and
against the host's own Cholesky inverse, and the two-level solve with the
device-built coarse space against the host-built one (CFD_COARSE_HOST=1)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rel_l2
from test_coarse_host import _hats, _laplace7

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 63, 64, 65, 200, 343])
def test_device_spd_inverse_matches_numpy(n):
    import cfdfs
    rng = np.random.default_rng(n)
    B = rng.standard_normal((n, n))
    A = B @ B.T + n * np.eye(n)
    inv = cfdfs.spd_inverse(A)
    assert rel_l2(inv, np.linalg.inv(A)) < 1e-12
    assert np.array_equal(inv, inv.T)


def test_device_inverse_of_coarse_matrix_matches_host():
    """Zc = P^T Z P of a 25^3 grid (343 coarse nodes, a shifted Laplacian):
    the device inverse against the host build's."""
    import cfdfs
    dims = (25, 25, 25)
    Z = _laplace7(dims, 0.05)
    Z.sort_indices()
    cd, inv_host = cfdfs.coarse_inverse(dims, Z.indptr.astype(np.int32), Z.indices.astype(np.int32), Z.data)
    P = sp.kron(_hats(dims[2]), sp.kron(_hats(dims[1]), _hats(dims[0]))).tocsr()
    inv_dev = cfdfs.spd_inverse((P.T @ Z @ P).toarray())
    assert rel_l2(inv_dev, inv_host) < 1e-10


def test_not_positive_definite_is_reported():
    import cfdfs
    A = np.eye(70)
    A[40, 40] = -1.0
    with pytest.raises(cfdfs.CfdError) as ei:
        cfdfs.spd_inverse(A)
    assert ei.value.code == cfdfs.CFD_E_NONFINITE


def test_twolevel_run_device_coarse_matches_host_coarse(tmp_path):
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c16.inp"), meshgen.CavitySpec(16, re=400, dt=0.005, steps=4))
    out = []
    for host in (False, True):
        if host:
            os.environ["CFD_COARSE_HOST"] = "1"
        try:
            s = cfdfs.Solver(device=0, precision=cfdfs.MIXED, precond=cfdfs.PC_TWOLEVEL)
        finally:
            os.environ.pop("CFD_COARSE_HOST", None)
        s.load(deck)
        s.step0()
        st = s.run(4)
        out.append((st, *s.state()))
        s.close()
    (sa, Ua, Pa), (sb, Ub, Pb) = out
    assert sa.subiters == sb.subiters and abs(sa.cg_iters - sb.cg_iters) <= sa.subiters
    assert rel_l2(Ua, Ub) < 1e-5 and rel_l2(Pa, Pb) < 1e-5


@pytest.mark.parametrize("case", ["cavity", "duct", "laplace65", "laplace_ragged"])
def test_device_coarse_matrix_is_bit_identical(case, tmp_path, oracle_mod):
    """The Galerkin product on the device (galerkin.cu) against the host
    build: the same sums in the same order, so the same bits."""
    import cfdfs
    from cfdfs import meshgen
    if case in ("cavity", "duct"):
        if case == "cavity":
            deck = meshgen.write_cavity(str(tmp_path / "c.inp"), meshgen.CavitySpec(12, re=100, dt=0.01, steps=2))
            dims = (13, 13, 13)
        else:
            deck = meshgen.write_duct(str(tmp_path / "d.inp"), n_cross=4, n_axial=24, steps=2, dt=0.01)
            dims = meshgen.duct_grid_dims(4, 24)
        o = oracle_mod.Oracle(deck)
        o.step0()
        Z = o.csr("Z").tocsr()
        o.close()
    else:
        dims = (65, 65, 65) if case == "laplace65" else (29, 21, 17)
        Z = _laplace7(dims, 0.05)
        Z.sort_indices()
        rng = np.random.default_rng(7)
        Z.data = Z.data * (1.0 + 1e-3 * rng.standard_normal(Z.data.size))
    rp, cl = Z.indptr.astype(np.int32), Z.indices.astype(np.int32)
    cd_h, zc_h = cfdfs.coarse_matrix(dims, rp, cl, Z.data)
    cd_d, zc_d = cfdfs.coarse_matrix(dims, rp, cl, Z.data, device=0)
    assert cd_h == cd_d
    assert np.array_equal(zc_h, zc_d)


def test_device_coarse_matrix_rejects_a_fine_lattice(tmp_path, oracle_mod):
    """A lattice finer than Z's reach (spacing 1.5 voxels against a matrix
    that couples nodes two voxels apart) leaves rows reaching more than 3
    coarse nodes per axis: the device build reports it, the host build
    still works."""
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c.inp"), meshgen.CavitySpec(6, re=100, dt=0.01, steps=2))
    dims = (7, 7, 7)
    o = oracle_mod.Oracle(deck)
    o.step0()
    Z = o.csr("Z").tocsr()
    o.close()
    rp, cl = Z.indptr.astype(np.int32), Z.indices.astype(np.int32)
    with pytest.raises(cfdfs.CfdError):
        cfdfs.coarse_matrix(dims, rp, cl, Z.data, spacing=1.5, device=0)
    cd, zc = cfdfs.coarse_matrix(dims, rp, cl, Z.data, spacing=1.5)
    assert np.array_equal(zc, zc.T)
