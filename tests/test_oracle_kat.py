"""Known-answer tests of the CPU oracle (the checker), from the mathematics of
the hex27/hex8 discretisation and the reference's coupling rules.  The
reference ships no tests or golden outputs, so these pin the oracle."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import REFERENCE_DECK

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sizes.json")


def test_shape_functions(decks, oracle_mod):
    for key in ("c1", "c1_27"):
        o = oracle_mod.Oracle(decks[key])
        b = o.basis()
        # partition of unity and zero-sum derivatives at every Gauss point
        assert np.allclose(b["Sv"].sum(axis=1), 1.0, atol=1e-14)
        assert np.allclose(b["Sp"].sum(axis=1), 1.0, atol=1e-14)
        assert np.allclose(b["dSv"].sum(axis=1), 0.0, atol=1e-13)
        assert np.allclose(b["dSp"].sum(axis=1), 0.0, atol=1e-14)
        # weights integrate the reference cube volume 8
        assert abs(b["gqw"].sum() - 8.0) < 1e-13
        # Kronecker property of the 27 nodal functions at the nodes
        o.close()


def test_element_volumes_and_mass(decks, oracle_mod):
    o = oracle_mod.Oracle(decks["graded"])
    gw = o.basis()["gqw"]
    vol = (o.detj() * gw[None, :]).sum(axis=1)
    assert abs(vol.sum() - 1.0) < 1e-12          # unit cube
    assert (vol > 0).all()
    o.step0()
    md = o.vec("MdOrig")[: o.NN]
    assert abs(md.sum() - 1.0) < 1e-12           # sum of lumped mass = |domain|
    assert (md > 0).all()
    o.close()


def test_operator_identities(decks, oracle_mod):
    o = oracle_mod.Oracle(decks["perturbed"])
    o.step0()
    K = o.csr("K")
    assert np.abs(K @ np.ones(o.NN)).max() < 1e-13 * np.abs(K.data).max()   # K 1 = 0
    assert abs(K - K.T).max() < 1e-15 * np.abs(K.data).max()
    Z = o.csr("Z")
    assert abs(Z - Z.T).max() <= 1e-14 * np.abs(Z.data).max()
    ev = np.linalg.eigvalsh(Z.toarray())
    assert ev.min() > 0                                               # SPD (pin applied)
    # G^T u for a constant field equals the boundary flux -int_dOmega Sp u.n
    G = [o.csr(g) for g in ("G1", "G2", "G3")]
    for d in range(3):
        s = np.asarray(G[d].sum(axis=0)).ravel()
        assert abs(s.sum()) < 1e-12                                   # total flux of a constant = 0
    o.close()


@pytest.mark.parametrize("key", ["c1", "c1_27"])
def test_convection_identities(decks, oracle_mod, key):
    """R1 = -A(Un) UnpHalf_prev with A_ij = sum_k Sv_i (u . grad Sv_j) detJ w
    (calculateMatrixA, blascoCodinaHuerta.cpp:3520-3685), per component:
    - a constant field has no convective derivative (A 1 = 0, because the
      gradients of the 27 shape functions sum to zero);
    - R1 is linear in UnpHalf_prev;
    - with u constant and x zero on the boundary, x . A x = 1/2 sum of
      u . grad(x^2) over the Gauss points vanishes: along each axis the
      tensor Gauss rule integrates the derivative of the polynomial x^2
      exactly, and the two elements of a shared face evaluate it at the same
      face points, so the element sums telescope to the boundary, where x
      is zero.  This holds for NGP 8 and 27 alike."""
    o = oracle_mod.Oracle(decks[key])
    o.step0()
    NN = o.NN
    X = o.coord()
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    o.set_vec("Un", np.concatenate([np.sin(np.pi * x) * y, np.cos(np.pi * y) * z, x * y * z]))
    rng = np.random.default_rng(7)

    def conv(v):
        o.set_vec("UnpHalf_prev", v)
        return o.convect()

    v1, v2 = rng.standard_normal(3 * NN), rng.standard_normal(3 * NN)
    r1, r2 = conv(v1), conv(v2)
    scale = np.abs(r1).max()
    assert scale > 0
    assert np.abs(conv(np.ones(3 * NN))).max() < 1e-13 * scale
    r12 = conv(2.0 * v1 - 3.0 * v2)
    assert np.abs(r12 - (2.0 * r1 - 3.0 * r2)).max() < 1e-12 * np.abs(r12).max()

    u = np.array([0.3, -0.5, 0.7])
    o.set_vec("Un", np.repeat(u, NN))
    bc = o.bcnodes()[:, 0]
    xv = rng.standard_normal(3 * NN)
    for d in range(3):
        xv[d * NN + bc] = 0.0
    r = conv(xv)
    for d in range(3):
        xd, rd = xv[d * NN:(d + 1) * NN], r[d * NN:(d + 1) * NN]
        assert abs(xd @ rd) < 1e-12 * np.linalg.norm(xd) * np.linalg.norm(rd)
    o.close()


def test_linear_fields_are_integrated_exactly(decks, oracle_mod):
    """A velocity or pressure field that is linear in the coordinates is
    represented exactly by the hex27 / hex8 spaces of straight-sided
    elements (mid-nodes at the corner averages), and the Gauss rule integrates
    the products below exactly, even on the non-affine perturbed mesh:
    - x.K x = nu |a|^2 |Omega| for x = a.X (K = nu int grad Sv . grad Sv);
    - sum_i X_d,i (G_d p)_i = -(1/rho) int p for p = b.X
      (G_d = -(1/rho) int Sp_j d_d Sv_i, and sum_i X_d,i Sv_i = X_d)."""
    a = np.array([0.3, 0.2, -0.5])
    b = np.array([0.7, -0.4, 0.25])
    for key in ("perturbed", "graded"):
        o = oracle_mod.Oracle(decks[key])
        o.step0()
        X = o.coord()
        gw = o.basis()["gqw"]
        vol = float((o.detj() * gw[None, :]).sum())
        x = X @ a
        K = o.csr("K")
        assert abs(x @ (K @ x) - o.viscosity * (a @ a) * vol) < 1e-12 * o.viscosity * vol
        # int p over the domain from the hex8 interpolation at the Gauss points
        bas = o.basis()
        conn = o.ltog()[:, :8]
        p = X[: o.NNp] @ b
        p_gp = p[conn] @ bas["Sp"].T                   # NE x NGP
        int_p = float((p_gp * o.detj() * gw[None, :]).sum())
        for d, name in enumerate(("G1", "G2", "G3")):
            G = o.csr(name)
            lhs = X[:, d] @ (G @ p)
            assert abs(lhs + int_p / o.density) < 1e-12 * max(1.0, abs(int_p)), (key, name, lhs, int_p)
        o.close()


def test_sizes_against_formulas(decks, oracle_mod):
    golden = json.load(open(GOLDEN))
    o = oracle_mod.Oracle(decks["c1"])
    o.step0()
    g = golden["c1_8"]
    assert (o.NN, o.NNp, o.nnzK, o.nnzG, o.nnzZ, o.nbc, o.ncolors) == \
        (g["NN"], g["NNp"], g["nnzK"], g["nnzG"], g["nnzZ"], g["nBCnodes"], g["colors"])
    assert o.zero_p == g["zeroP"] and o.mon == g["monPoint"]
    o.close()


@pytest.mark.skipif(not os.path.exists(REFERENCE_DECK), reason="reference deck not present")
def test_shipped_deck_counts(oracle_mod):
    golden = json.load(open(GOLDEN))["shipped_30"]
    o = oracle_mod.Oracle(REFERENCE_DECK)
    assert (o.NE, o.NCN, o.NN, o.NNp, o.nnzK, o.nnzG) == \
        (golden["NE"], golden["NCN"], golden["NN"], golden["NNp"], golden["nnzK"], golden["nnzG"])
    assert o.nbc == golden["nBCnodes"] and o.ncolors == 8
    o.close()


def test_bc_ownership(decks, oracle_mod):
    """Later faces overwrite earlier ones: the lid (BC 2, listed last) owns
    its edges and corners."""
    o = oracle_mod.Oracle(decks["c1"])
    bc = o.bcnodes()
    xyz = o.coord()
    lid = bc[xyz[bc[:, 0], 2] == 1.0]
    assert (lid[:, 1] == 1).all()
    assert len(bc) == 17 ** 3 - 15 ** 3
    o.close()


def test_step_count_trap():
    from cfdfs.meshgen import steps_for, t_final_for_steps
    assert steps_for(0.01, 0.2) == 20
    assert steps_for(0.005, 1.0) == 200
    assert steps_for(0.002, 0.2) == 100
    assert steps_for(0.005, 1.5) == 301
    assert steps_for(0.005, t_final_for_steps(0.005, 300)) == 300


def test_cg_oracle_solves(decks, oracle_mod):
    o = oracle_mod.Oracle(decks["c1"])
    o.step0()
    Z = o.csr("Z")
    rng = np.random.default_rng(0)
    b = rng.standard_normal(o.NNp)
    o.set_cg(1e-10, 1000, 0)
    x, st = o.cg(b)
    assert st[2] == 0
    assert np.linalg.norm(b - Z @ x) <= 1.01e-10 * np.linalg.norm(b)
    o.close()


def test_oracle_run_deterministic(decks, oracle_mod):
    """Fixed reduction chunking: the same result with 1 and 4 threads."""
    outs = []
    for th in (1, 4):
        o = oracle_mod.Oracle(decks["c1"], threads=th)
        o.step0()
        o.run(3)
        outs.append((o.vec("Un"), o.vec("Pn")))
        o.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
