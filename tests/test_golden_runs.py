"""The golden end states of full-size oracle runs (tests/golden/*.npz, made by
tests/golden/make_run_goldens.py) on the CPU: their subsamples fit the
generated decks, the cavity's state keeps the mirror symmetry of the
problem, and the duct's inlet profile is the same whether it is taken from
the oracle's mesh or from the product's host mesh."""
import importlib.util
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _gen():
    spec = importlib.util.spec_from_file_location("make_run_goldens",
                                                  os.path.join(HERE, "golden", "make_run_goldens.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("case", ["c2_cavity32", "c3_cavity64", "duct_24x160"])
def test_golden_file_fits_its_deck(case, tmp_path):
    from cfdfs import HostMesh
    g = _gen()
    gd = np.load(os.path.join(HERE, "golden", f"{case}.npz"))
    h = HostMesh(g.deck_for(case, str(tmp_path)))
    assert len(gd["u_sub"]) == math.ceil(3 * h.NN / int(gd["u_stride"]))
    assert len(gd["p_sub"]) == math.ceil(h.NNp / int(gd["p_stride"]))
    assert int(gd["steps"]) == g.CASES[case]["steps"]
    assert np.all(np.isfinite(gd["u_sub"])) and np.all(np.isfinite(gd["p_sub"]))
    h.close()


@pytest.mark.parametrize("case", ["c2_cavity32", "c3_cavity64"])
def test_cavity_golden_keeps_mirror_symmetry(case):
    """The lid moves along x, so the flow is symmetric about the plane
    y = 1/2, where v vanishes: v at the monitor node (the cube centre) is
    zero to rounding while u and w are not."""
    gd = np.load(os.path.join(HERE, "golden", f"{case}.npz"))
    u, v, w, _ = gd["mon"]
    assert abs(v) < 1e-12 * max(abs(u), abs(w))
    assert abs(u) > 1e-3


def test_inlet_profile_same_on_both_meshes(decks, oracle_mod):
    from cfdfs import HostMesh, meshgen
    o = oracle_mod.Oracle(decks["duct_small"])
    h = HostMesh(decks["duct_small"])
    n_o, uvw_o = meshgen.duct_inlet_profile(o)
    n_h, uvw_h = meshgen.duct_inlet_profile(h)
    assert len(n_o) > 0
    assert np.array_equal(n_o, n_h) and np.array_equal(uvw_o, uvw_h)
    h.close()
    o.close()
