"""The bent-duct deck generator (cfdfs.meshgen) against the geometry it is
specified with: a 1 x 1 square section, a straight inlet leg of length 3
along +x, a 90-degree bend of centreline radius 2 about the z axis, a
straight outlet leg of length 3 along +y, and a parabolic inlet of peak 1.0.

The mesh's volume, integrated by the oracle (Gauss rule on the trilinear
element maps, exact for their Jacobians), has a closed form: each bend
segment of angle d is a prism whose section is the trapezoid between two
chords, of area R sin d, so the volume is 2 * 3 + n_bend * 2 sin(pi / (2
n_bend)), which tends to 6 + pi."""
import math

import numpy as np
import pytest


@pytest.mark.parametrize("n_cross,n_axial", [(4, 40), (2, 61)])
def test_duct_volume_and_planes(tmp_path, oracle_mod, n_cross, n_axial):
    from cfdfs import meshgen
    deck = meshgen.write_duct(str(tmp_path / "duct.inp"), n_cross=n_cross, n_axial=n_axial, steps=1, dt=0.01)
    o = oracle_mod.Oracle(deck)
    gw = o.basis()["gqw"]
    vol = float((o.detj() * gw[None, :]).sum())
    n1 = max(1, round(n_axial * 3.0 / (6.0 + math.pi)))
    n2 = n_axial - 2 * n1
    expected = 6.0 + n2 * 2.0 * math.sin(0.5 * math.pi / n2)
    # the deck stores coordinates to 9 decimals: volume exact to about 1e-10
    assert abs(vol - expected) < 1e-8 * expected
    assert abs(vol - (6.0 + math.pi)) < 0.02
    X = o.coord()
    corners = X[: o.NCN]
    # inlet plane x = 0, outlet plane y = 5 (= radius + leg), section 1 x 1
    assert corners[:, 0].min() == pytest.approx(0.0, abs=1e-14)
    assert corners[:, 1].max() == pytest.approx(5.0, abs=1e-12)
    assert corners[:, 2].min() == pytest.approx(-0.5) and corners[:, 2].max() == pytest.approx(0.5)
    o.close()


def test_duct_inlet_profile(tmp_path):
    """Parabolic inlet u = (1 - (2y)^2)(1 - (2z)^2) along +x: peak 1.0 at the
    section centre, zero on the walls, on the inlet plane only."""
    from cfdfs import HostMesh, meshgen
    deck = meshgen.write_duct(str(tmp_path / "duct.inp"), n_cross=4, n_axial=20, steps=1, dt=0.01)
    h = HostMesh(deck)
    nodes, uvw = meshgen.duct_inlet_profile(h)
    X = h.coord()[nodes]
    h.close()
    assert np.all(np.abs(X[:, 0]) < 1e-14)
    assert uvw[:, 0].max() == pytest.approx(1.0, abs=1e-15)
    assert np.all(uvw[:, 1:] == 0.0) and np.all(uvw[:, 0] >= 0.0)
    y, z = X[:, 1], X[:, 2]
    assert np.allclose(uvw[:, 0], (1 - 4 * y * y) * (1 - 4 * z * z), atol=1e-15)
    # wall rim nodes of the inlet belong to the walls (listed after the inlet)
    assert np.all((np.abs(y) < 0.5 - 1e-12) & (np.abs(z) < 0.5 - 1e-12))
