"""Parity with the reference itself, on the CPU.

The fixtures ``tests/golden/ref_<case>.npz`` hold what the reference's own
solver (fractionalStep/Cpp/blascoCodinaHuerta.cpp, compiled unmodified
against the stand-in MKL and CSparse of ``oracle/refshim``;
``tests/golden/make_ref_goldens.py``) printed and wrote for each case.  Here:

* the oracle, run with the reference's solve (Jacobi-PCG from x0 = 0 to
  ||r|| <= 1e-6 ||b||, the MKL dcg settings of blascoCodinaHuerta.cpp:
  3998-4018), must reproduce the final fields to 1e-9 relative, the CG
  iteration count of every pressure solve and every monitor row exactly;
* the Tecplot text that the oracle and the product's host code write must
  carry the reference's node numbering and element-to-node map (hashes of
  the coordinate and connectivity text, bit for bit).
"""
import os
import tempfile

import numpy as np
import pytest

import ref_cases
from conftest import GOLDEN

CASES = list(ref_cases.CASES)


def _deck(name, tmp):
    path = os.path.join(tmp, name + ".inp")
    if name == "shipped_ne27000":
        src = ref_cases.shipped_deck_path()
        if src is None:
            pytest.skip("reference deck not found (set CFD_REFERENCE_DIR)")
        text = ref_cases.shipped_deck_text(src)
    else:
        text = ref_cases.deck_text(name)
    with open(path, "w") as f:
        f.write(text)
    return path, text


def _mon_norm(text):
    # the sign of a printed zero follows rounding noise (v on the cavity's
    # symmetry plane is ~1e-17 of either sign in both codes)
    return text.replace("-0.00000", " 0.00000")


@pytest.mark.parametrize("name", CASES + ["shipped_ne27000"])
def test_oracle_matches_reference(oracle_mod, name):
    fix = ref_cases.load_fixture(name, GOLDEN)
    with tempfile.TemporaryDirectory() as tmp:
        path, text = _deck(name, tmp)
        assert ref_cases.sha256_text(text) == str(fix["deck_sha256"]), "deck generator changed"
        o = oracle_mod.Oracle(path)
        o.set_cg(rtol=ref_cases.REF_CG_RTOL, maxit=ref_cases.REF_CG_MAXIT, warm=0)
        o.step0()
        o.run(-1)
        cg, mon = o.logs()
        dat_path = os.path.join(tmp, name + ".dat")
        assert o.write_tecplot(dat_path, name) == 0
        dat = ref_cases.parse_dat(open(dat_path).read())
        o.close()
    # numbering, coordinates and connectivity, bit for bit
    assert dat["zone"] == str(fix["zone"])
    assert dat["xyz_sha"] == str(fix["xyz_sha"])
    assert dat["conn_sha"] == str(fix["conn_sha"])
    # the CG iterations of every pressure solve, the sub-iteration count of
    # every step (monitor "Iter" column) and the steady-state stop
    assert np.array_equal(cg, fix["cg_iters"])
    assert mon.shape == fix["mon"].shape
    assert np.array_equal(mon[:, :2], fix["mon"][:, :2])
    ours = [_mon_norm(ref_cases.monitor_text(*row)) for row in mon]
    assert ours == [_mon_norm(t) for t in fix["mon_text"]]
    # final fields
    d = ref_cases.compare_summary(fix, dat["uvwp"])
    for field, r in d.items():
        for k, v in r.items():
            assert v <= 1e-9, (field, k, v)


@pytest.mark.parametrize("name", ["c1", "graded", "perturbed", "duct_small", "c16", "shipped_ne27000"])
def test_product_numbering_matches_reference(oracle_mod, name):
    """The product's host preprocessing (cfdh_load, C++) and its Tecplot
    writer give the reference's node numbering and element map."""
    from cfdfs import HostMesh
    fix = ref_cases.load_fixture(name, GOLDEN)
    with tempfile.TemporaryDirectory() as tmp:
        path, _ = _deck(name, tmp)
        h = HostMesh(path)
        # the field values do not enter the hashes; zeros will do
        out = os.path.join(tmp, "p.dat")
        h.write_tecplot(np.zeros(3 * h.NN), np.zeros(h.NNp), out, name)
        dat = ref_cases.parse_dat(open(out).read())
        h.close()
    assert dat["zone"] == str(fix["zone"])
    assert dat["xyz_sha"] == str(fix["xyz_sha"])
    assert dat["conn_sha"] == str(fix["conn_sha"])


def test_fixture_steady_case_stops_early():
    """The steady deck asks for 100 steps; the reference's maxAcc test
    (blascoCodinaHuerta.cpp:3048-3061, max |Unp1 - Un| / dt <= converge)
    stopped it earlier, and its last maxAcc is below the criterion."""
    fix = ref_cases.load_fixture("steady", GOLDEN)
    mon = fix["mon"]
    assert len(mon) < 100
    assert mon[-1, 7] <= 0.05 < mon[-2, 7]
