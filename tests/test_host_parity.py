"""The product's host preprocessing (C++, cfdh_* entry points) against the
oracle's restatement of the reference's own algorithms: identical node
numbering, coordinates, BC nodes, monitor node and CSR patterns (bit-exact)."""
import os

import numpy as np
import pytest

from conftest import REFERENCE_DECK


def _compare(path, oracle_mod):
    from cfdfs import HostMesh
    o = oracle_mod.Oracle(path)
    o.step0()
    h = HostMesh(path)
    assert (h.NE, h.NCN, h.NN, h.NNp) == (o.NE, o.NCN, o.NN, o.NNp)
    assert np.array_equal(h.ltog(), o.ltog())
    assert np.array_equal(h.coord(), o.coord())          # bit-exact coordinates
    assert np.array_equal(h.bcnodes(), o.bcnodes())
    assert h.mon == o.mon and h.zero_p == o.zero_p
    for which in ("K", "G", "Z"):
        rp_h, col_h = h.pattern(which)
        rp_o, col_o = o.pattern(which)
        assert np.array_equal(rp_h, rp_o), which
        assert np.array_equal(col_h, col_o), which
    # G^T is the transpose of G
    rp_g, col_g = h.pattern("G")
    rp_t, col_t = h.pattern("GT")
    import scipy.sparse as sp
    Gs = sp.csr_matrix((np.ones(len(col_g)), col_g, rp_g), shape=(h.NN, h.NNp))
    Ts = Gs.T.tocsr()
    Ts.sort_indices()
    assert np.array_equal(Ts.indptr, rp_t) and np.array_equal(Ts.indices, col_t)
    h.close()
    o.close()


@pytest.mark.parametrize("key", ["c1", "graded", "perturbed", "duct_small"])
def test_host_preprocessing_matches_oracle(decks, oracle_mod, key):
    _compare(decks[key], oracle_mod)


@pytest.mark.skipif(not os.path.exists(REFERENCE_DECK), reason="reference deck not present")
def test_host_preprocessing_shipped_deck(oracle_mod):
    _compare(REFERENCE_DECK, oracle_mod)


def test_bad_decks_rejected(tmp_path, decks):
    from cfdfs import HostMesh, CfdError
    good = open(decks["c1"]).read()
    cases = {
        "truncated": good[: len(good) // 3],
        "bad_corner": good.replace("\n     1        1        2", "\n     1        0        2", 1),
        "not_hex": good.replace("NENv     : 27", "NENv     : 8"),
        "empty": "",
    }
    for name, text in cases.items():
        p = tmp_path / f"{name}.inp"
        p.write_text(text)
        with pytest.raises(CfdError):
            HostMesh(str(p))
    with pytest.raises(CfdError):
        HostMesh(str(tmp_path / "missing.inp"))


def _edit_after(text, header, fn):
    """The deck with fn applied to the first data line after the line that
    starts with header (skipping the ==== separator lines)."""
    lines = text.split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith(header)) + 1
    while lines[i].startswith("===="):
        i += 1
    lines[i] = fn(lines[i])
    return "\n".join(lines)


def test_out_of_range_values_rejected(tmp_path, decks):
    """Values that would index outside the mesh or break the time loop are
    rejected on the host with a message, before anything reaches the device:
    a velocity BC face outside 1..6, a BC number beyond nBC, a zero-pressure
    node beyond the corner nodes, dt <= 0, and an NGP other than 1, 8, 27."""
    from cfdfs import HostMesh, CfdError
    good = open(decks["c1"]).read()
    HostMesh(decks["c1"]).close()
    hdr = "Velocity BC (Elem# Face# BC#)"
    cases = {
        "face": (_edit_after(good, hdr, lambda l: " ".join(l.split()[:1] + ["9"] + l.split()[2:])),
                 "velocity BC face out of range"),
        "bc_id": (_edit_after(good, hdr, lambda l: " ".join(l.split()[:2] + ["5"])),
                  "velocity BC face out of range"),
        "zero_p": (_edit_after(good, "Node number where pressure", lambda l: "100000"),
                   "zero-pressure node out of range"),
        "dt": ("\n".join(("dt       : 0.0" if l.startswith("dt ") else l) for l in good.split("\n")),
               "dt must be > 0"),
        "ngp": ("\n".join(("NGP      : 4" if l.startswith("NGP") else l) for l in good.split("\n")),
                "NGP must be 1, 8 or 27"),
    }
    for name, (text, msg) in cases.items():
        assert text != good, name
        p = tmp_path / f"{name}.inp"
        p.write_text(text)
        with pytest.raises(CfdError, match=msg):
            HostMesh(str(p))


def test_number_forms_read_as_strtod(tmp_path):
    """The deck reader takes numbers in the forms the reference's istream
    extraction (strtol / strtod) accepts: the same corner coordinates written
    with a leading '+', an exponent, a hexadecimal mantissa, no integer or no
    fraction digits, and node numbers with a leading '+', give bit-identical
    coordinates and the same mesh."""
    from cfdfs import HostMesh, meshgen
    path = meshgen.write_cavity(str(tmp_path / "c2.inp"), meshgen.CavitySpec(2, re=100, dt=0.01, steps=2, ngp=8))
    text = open(path).read()
    forms = {0.0: ["+0.0", "0e5", "0x0p0", ".0", "0."], 0.5: ["+0.5", "5e-1", "0x1p-1", ".5", "+.5E0"],
             1.0: ["1.", "+1", "1e0", "0X1P0", "10e-1"]}
    lines = text.split("\n")
    first = next(k for k, l in enumerate(lines) if l.startswith("Corner Node No")) + 1
    for k in range(27):
        f = lines[first + k].split()
        out = ["+" + f[0] if k % 2 else f[0]]
        for c, v in enumerate(f[1:]):
            alts = forms[float(v)]
            out.append(alts[(k + c) % len(alts)])
        lines[first + k] = "   ".join(out)
    alt = tmp_path / "c2_forms.inp"
    alt.write_text("\n".join(lines))
    a, b = HostMesh(path), HostMesh(str(alt))
    assert a.coord().tobytes() == b.coord().tobytes()
    assert np.array_equal(a.ltog(), b.ltog()) and np.array_equal(a.bcnodes(), b.bcnodes())
    a.close()
    b.close()


@pytest.mark.parametrize("key", ["c1", "graded", "perturbed", "duct_small"])
def test_element_colouring_conflict_free(decks, key):
    """The deterministic mode's colouring (one colour per launch, plain adds):
    every element exactly once, and no two elements of a colour share any of
    their 27 nodes (corners, edge and face mid-nodes, centre)."""
    from cfdfs import HostMesh
    h = HostMesh(decks[key])
    order, off = h.element_colors()
    assert np.array_equal(np.sort(order), np.arange(h.NE))
    assert off[0] == 0 and off[-1] == h.NE and np.all(np.diff(off) > 0)
    ltog = h.ltog()
    for c in range(len(off) - 1):
        els = order[off[c]:off[c + 1]]
        assert np.all(np.diff(els) > 0)  # ascending inside a colour: a fixed order
        nodes = ltog[els].ravel()
        assert len(np.unique(nodes)) == len(nodes), f"colour {c} shares a node"
    # a structured hex mesh needs the 8 colours of the parity classes
    if key in ("c1", "graded", "perturbed"):
        assert len(off) - 1 == 8
    h.close()
