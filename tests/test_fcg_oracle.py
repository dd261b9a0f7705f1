"""The direction windows of flexible CG (oracle/fcg_oracle.py, the NumPy
restatement of csrc/cuda/fcg.cu) on the pressure matrix Z of the 8^3 cavity,
with Jacobi as the fixed preconditioner and a nonlinear head (the role the
U-Net plays) in the first iterations.

The anchored window keeps the head's directions for the whole solve. It is
CG deflated by their span, so every direction stays Z-conjugate to all
earlier ones, and it needs the iterations of full orthogonalisation. A ring
window forgets the head's directions and loses that conjugacy.  Tolerances:
conjugacy (|(p_i, Z p_j)| normalised) below 1e-7 where the theory gives
exact conjugacy, above 1e-2 where it does not; iteration counts equal to
full orthogonalisation within one."""
import numpy as np
import pytest

import fcg_oracle as F


@pytest.fixture(scope="module")
def system(decks, oracle_mod):
    o = oracle_mod.Oracle(decks["c1"])
    o.step0()
    Z = o.csr("Z")
    b = np.random.default_rng(3).standard_normal(Z.shape[0])
    b[o.zero_p] = 0.0
    o.close()
    return Z, b, 1.0 / Z.diagonal()


def _precond(dinv, head_iters):
    def head(r):
        z = dinv * r
        # nonlinear in r, still a descent direction: z.r > 0
        return z + 0.8 * z ** 3 / np.max(np.abs(z)) ** 2

    return lambda r, it: head(r) if it < head_iters else dinv * r


def test_slot_rule():
    assert [F.fcg_slot(i, 2, 1) for i in range(5)] == [0, 1, 1, 1, 1]
    assert [F.fcg_slot(i, 4, 3) for i in range(6)] == [0, 1, 2, 3, 3, 3]
    assert [F.fcg_slot(i, 4, 0) for i in range(6)] == [0, 1, 2, 3, 0, 1]


@pytest.mark.parametrize("head", [1, 3])
def test_anchored_window_is_deflated_cg(system, head):
    Z, b, dinv = system
    pc = _precond(dinv, head)
    xa, ia, da = F.fcg(Z, b, pc, m=head + 1, anchor=head, rtol=1e-10)
    xf, i_full, df = F.fcg(Z, b, pc, m=1000, rtol=1e-10)
    assert np.linalg.norm(b - Z @ xa) <= 1.01e-10 * np.linalg.norm(b)
    assert F.conjugacy(Z, da) < 1e-7
    assert abs(ia - i_full) <= 1
    assert np.linalg.norm(xa - xf) <= 1e-8 * np.linalg.norm(xf)


@pytest.mark.parametrize("m", [1, 4])
def test_ring_window_loses_the_head(system, m):
    Z, b, dinv = system
    x, its, dirs = F.fcg(Z, b, _precond(dinv, 1), m=m, rtol=1e-10)
    assert np.linalg.norm(b - Z @ x) <= 1.01e-10 * np.linalg.norm(b)
    assert F.conjugacy(Z, dirs) > 1e-2
    _, i_anchor, _ = F.fcg(Z, b, _precond(dinv, 1), m=2, anchor=1, rtol=1e-10)
    assert its >= i_anchor


def test_linear_head_is_cg(system):
    """With the fixed preconditioner from the first iteration on, the anchored
    window is plain preconditioned CG: same iterations, same solution."""
    Z, b, dinv = system
    pc = lambda r, it: dinv * r
    xa, ia, _ = F.fcg(Z, b, pc, m=2, anchor=1, rtol=1e-10)
    xc, ic, _ = F.fcg(Z, b, pc, m=1, rtol=1e-10)
    assert ia == ic
    assert np.linalg.norm(xa - xc) <= 1e-8 * np.linalg.norm(xc)
