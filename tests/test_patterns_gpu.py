"""The operator patterns built on the device (csrc/cuda/patterns.cu, the
solver's load path) against the host build (build_patterns, the path of
cfdh_load that the host-parity tests pin to the reference's numbering): the
row pointers and columns of K, G, G^T and Z must be identical, and G^T's
slot map must point at the matching entries of G."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1", "graded", "perturbed", "duct_small"])
def test_device_patterns_equal_host_patterns(decks, name):
    import cfdfs
    h = cfdfs.HostMesh(decks[name])
    s = cfdfs.Solver(device=0)
    s.load(decks[name])
    s.step0()
    for which in ("K", "G", "GT", "Z"):
        rp_h, col_h = h.pattern(which)
        rp_d, col_d, _ = s.matrix(which)
        assert np.array_equal(rp_d, rp_h), which
        assert np.array_equal(col_d, col_h), which
    # values of G^T are G's through gt_pos: the transposed products agree
    rp_g, col_g, g = s.matrix("G")
    rp_t, col_t, gt = s.matrix("GT")
    nn = len(rp_g) - 1
    rows_g = np.repeat(np.arange(nn), np.diff(rp_g))
    G = {(int(r), int(c)): v for r, c, v in zip(rows_g, col_g, g[:, 0])}
    rows_t = np.repeat(np.arange(len(rp_t) - 1), np.diff(rp_t))
    for p, v, val in zip(rows_t[::97], col_t[::97], gt[::97, 0]):
        assert G[(int(v), int(p))] == val
    s.close()
    h.close()


def _device_pattern(s, which, nrows):
    """(rowptr, col) of the solver's operator, without values."""
    import ctypes as C
    import cfdfs
    nnz = C.c_longlong(0)
    w = cfdfs.MAT[which]
    assert s.L.cfd_download_matrix(s.h, w, C.byref(nnz), None, None, None) == 0
    rp = np.zeros(nrows + 1, dtype=np.int32)
    col = np.zeros(nnz.value, dtype=np.int32)
    assert s.L.cfd_download_matrix(s.h, w, C.byref(nnz), cfdfs._p(rp, C.c_int), cfdfs._p(col, C.c_int), None) == 0
    return rp, col


def test_device_patterns_of_the_64_cavity_equal_host_patterns(tmp_path):
    """The 64^3 benchmark deck (2.1 M velocity rows, 275 k pressure rows)."""
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c64.inp"), meshgen.CavitySpec(64, re=1000, dt=0.002, steps=2))
    h = cfdfs.HostMesh(deck)
    s = cfdfs.Solver(device=0)
    s.load(deck)
    for which in ("K", "G", "GT", "Z"):
        rp_h, col_h = h.pattern(which)
        rp_d, col_d = _device_pattern(s, which, len(rp_h) - 1)
        assert np.array_equal(rp_d, rp_h), which
        assert np.array_equal(col_d, col_h), which
    s.close()
    h.close()


def test_host_pattern_fallback_gives_the_same_run(decks):
    """CFD_HOST_PATTERNS=1 takes the host build (the fallback when a row has
    more candidates than the device build holds): the same operators and a
    bit-identical run in deterministic mode."""
    import os
    import cfdfs
    out = []
    for host in (True, False):
        os.environ["CFD_HOST_PATTERNS"] = "1" if host else "0"
        try:
            s = cfdfs.Solver(device=0, deterministic=1)
        finally:
            del os.environ["CFD_HOST_PATTERNS"]
        s.load(decks["graded"])
        s.step0()
        mats = [s.matrix(w) for w in ("K", "G", "GT", "Z")]
        s.run(3)
        out.append((mats, *s.state()))
        s.close()
    (ma, Ua, Pa), (mb, Ub, Pb) = out
    for a, b in zip(ma, mb):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert np.array_equal(Ua, Ub) and np.array_equal(Pa, Pb)
