"""Shared fixtures: generated input decks, the CPU oracle (checker) and the
product binding.  GPU tests are marked ``gpu``."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cfd-with-cuda_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, os.path.join(ROOT, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)

import ref_cases  # noqa: E402

# The reference's shipped 30^3 deck is not part of this repository: tests
# that read it find it under $CFD_REFERENCE_DIR and skip without it.
REFERENCE_DECK = os.path.join(os.environ.get("CFD_REFERENCE_DIR", "/nonexistent"), ref_cases.SHIPPED_REL)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


perturbed_box = ref_cases.perturbed_box


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
