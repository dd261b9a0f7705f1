"""Test infrastructure (the checker, never the product): a NumPy restatement
of the truncated flexible CG of the pressure solves,
cfd-with-cuda_b200/csrc/cuda/fcg.cu.

FCG(m) (Notay, "Flexible conjugate gradients", SIAM J. Sci. Comput. 22,
2000) orthogonalises each new direction, in the Z inner product, against
the directions in a window of stored ones:

- the ring: the last m directions (m = 1 is the Polak-Ribiere form, which is
  CG for a fixed symmetric preconditioner);
- the anchored window: the first a directions stay for the whole solve and
  every later direction is orthogonalised against them and its predecessor
  (m = a + 1).  With the first a directions from a nonlinear preconditioner
  and the rest from a fixed symmetric one, this is CG deflated by the span of
  the first a directions (Saad, Yeung, Erhel and Guyomarc'h, "A deflated
  version of the conjugate gradient algorithm", SIAM J. Sci. Comput. 21,
  2000): after the head, r is Z-orthogonal to that span, and every direction
  stays Z-orthogonal to all earlier ones.

One iteration, in the kernels' order and with their formulas:
  z = B(r); w = Z z
  beta_j = (z, q_j) / (p_j, q_j) for the stored slots j
  (p, q) = (z, w) - sum beta_j (z, q_j);  (p, r) = (z, r) - sum beta_j (p_j, r)
  alpha = (p, r) / (p, q)
  p = z - sum beta_j p_j;  q = w - sum beta_j q_j   (into slot fcg_slot(it))
  x += alpha p;  r -= alpha q
The reference has no counterpart (its pressure solver is Jacobi-PCG); this
file serves the tests of the windows only.
"""
from __future__ import annotations

import numpy as np


def fcg_slot(it: int, m: int, anchor: int) -> int:
    """Slot of direction it (0-based): the rule of fcg_slot in kernels.h."""
    if anchor > 0:
        return it if it < anchor else anchor
    return it % m


def fcg(Z, b, precond, m: int = 1, anchor: int = 0, rtol: float = 1e-10, maxit: int = 1000):
    """Solves Z x = b from x = 0.  precond(r, it) -> z is the preconditioner
    of iteration it (it may change from one iteration to the next).
    Returns (x, iterations, directions), directions = every p in order."""
    if anchor > 0 and m != anchor + 1:
        raise ValueError("the anchored window needs m = anchor + 1")
    n = b.shape[0]
    x = np.zeros(n)
    r = np.array(b, dtype=np.float64)
    P = [None] * m
    Q = [None] * m
    PQ = [0.0] * m
    bb = float(r @ r)
    dirs = []
    for it in range(maxit):
        z = precond(r, it)
        w = Z @ z
        nd = min(it, m)
        pq = float(z @ w)
        pr = float(z @ r)
        p = z.copy()
        q = w.copy()
        for j in range(nd):
            zq = float(z @ Q[j])
            bj = zq / PQ[j]
            pq -= bj * zq
            pr -= bj * float(P[j] @ r)
            p -= bj * P[j]
            q -= bj * Q[j]
        if not pq > 0.0:
            raise FloatingPointError("breakdown: the direction carries no descent")
        alpha = pr / pq
        k = fcg_slot(it, m, anchor)
        P[k], Q[k], PQ[k] = p, q, pq
        x += alpha * p
        r -= alpha * q
        dirs.append(p)
        if float(r @ r) <= rtol * rtol * bb:
            return x, it + 1, dirs
    return x, maxit, dirs


def conjugacy(Z, dirs) -> float:
    """Largest |(p_i, Z p_j)| / sqrt((p_i, Z p_i)(p_j, Z p_j)) over i != j."""
    D = np.stack(dirs, axis=1)
    G = D.T @ (Z @ D)
    d = np.sqrt(np.diag(G))
    C = np.abs(G) / np.outer(d, d)
    np.fill_diagonal(C, 0.0)
    return float(C.max())
