"""Shared fixtures: generated input decks, the CPU oracle (checker) and the
product binding.  GPU tests are marked ``gpu``."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cfd-with-cuda_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

REFERENCE_DECK = "/root/reference/inputFiles/lidDrivenCavity/lidDrivenCavity_NE27000.inp"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def perturbed_box(nx, ny, nz, amp, seed):
    """Corner nodes of an nx x ny x nz box with interior nodes moved by a
    seeded random offset (non-affine elements exercise the full Jacobian)."""
    from cfdfs import meshgen
    m = (nx + 1, ny + 1, nz + 1)
    k, j, i = np.meshgrid(np.arange(m[2]), np.arange(m[1]), np.arange(m[0]), indexing="ij")
    xyz = np.stack([i.ravel() / nx, j.ravel() / ny, k.ravel() / nz], axis=1).astype(np.float64)
    rng = np.random.default_rng(seed)
    interior = (i.ravel() > 0) & (i.ravel() < nx) & (j.ravel() > 0) & (j.ravel() < ny) & (k.ravel() > 0) & \
               (k.ravel() < nz)
    h = min(1.0 / nx, 1.0 / ny, 1.0 / nz)
    xyz[interior] += rng.uniform(-amp * h, amp * h, size=(interior.sum(), 3))
    xyz = np.round(xyz, 9)
    ek, ej, ei = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ei, ej, ek = ei.ravel(), ej.ravel(), ek.ravel()
    node = lambda a, b, c: a + m[0] * b + m[0] * m[1] * c
    conn = np.stack([node(ei, ej, ek), node(ei + 1, ej, ek), node(ei + 1, ej + 1, ek), node(ei, ej + 1, ek),
                     node(ei, ej, ek + 1), node(ei + 1, ej, ek + 1), node(ei + 1, ej + 1, ek + 1),
                     node(ei, ej + 1, ek + 1)], axis=1)
    eid = np.arange(nx * ny * nz) + 1
    faces = []
    for face, sel, bc in ((1, ek == 0, 1), (5, ei == 0, 1), (3, ei == nx - 1, 1), (2, ej == 0, 1),
                          (4, ej == ny - 1, 1), (6, ek == nz - 1, 2)):
        e = eid[sel]
        faces.append(np.stack([e, np.full_like(e, face), np.full_like(e, bc)], axis=1))
    return xyz, conn, np.concatenate(faces)


@pytest.fixture(scope="session")
def decks(tmp_path_factory):
    """Generated decks: name -> path."""
    from cfdfs import meshgen
    d = tmp_path_factory.mktemp("decks")
    out = {}
    out["c1"] = meshgen.write_cavity(str(d / "c1.inp"), meshgen.CavitySpec(8, re=100, dt=0.01, steps=20, ngp=8))
    out["c1_27"] = meshgen.write_cavity(str(d / "c1_27.inp"),
                                        meshgen.CavitySpec(8, re=100, dt=0.01, steps=20, ngp=27))
    # sub-iteration limit 2: every step ends with the loop run out
    out["c1_runout"] = meshgen.write_cavity(str(d / "c1_runout.inp"),
                                            meshgen.CavitySpec(8, re=100, dt=0.01, steps=5, ngp=8, max_iter=2))
    out["graded"] = meshgen.write_cavity(str(d / "graded.inp"),
                                         meshgen.CavitySpec(6, re=400, dt=0.005, steps=5, ngp=8, grading=1.5))
    xyz, conn, faces = perturbed_box(5, 4, 3, 0.2, seed=7)
    out["perturbed"] = meshgen.write_text(str(d / "perturbed.inp"), meshgen.deck_from_arrays(
        xyz, conn, faces, [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0)], zero_p_node1=3, ngp=8, dt=0.01, steps=5,
        viscosity=0.01))
    out["duct_small"] = meshgen.write_duct(str(d / "duct_small.inp"), n_cross=3, n_axial=16, steps=3, dt=0.01)
    return out


@pytest.fixture(scope="session")
def oracle_mod():
    import pyoracle
    pyoracle.build()
    return pyoracle
