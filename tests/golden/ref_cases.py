"""Reference-parity cases (TEST INFRASTRUCTURE).

The decks below are generated, so they can be rebuilt byte for byte on any
machine; ``make_ref_goldens.py`` ran the reference's own CPU solver
(fractionalStep/Cpp/blascoCodinaHuerta.cpp compiled unmodified against the
stand-in MKL and CSparse of ``oracle/refshim``) on each of them and stored
what it printed and wrote in ``ref_<case>.npz``.  The tests rebuild the deck,
check its hash against the one the fixture recorded, run the oracle or the
GPU path on it, and compare.

Also here: the readers of the reference's two outputs, the Tecplot file of
createTecplot (blascoCodinaHuerta.cpp:4249-4482) and the screen output of
timeLoop (the monitor table, blascoCodinaHuerta.cpp:2853-2854, 3091-3093, and
the "MKL_CG converged after N iterations." line of each pressure solve,
blascoCodinaHuerta.cpp:4032), and the field summary the fixtures store.
"""
from __future__ import annotations

import hashlib
import os
import re

import numpy as np

# Reference solve of these fixtures: MKL dcg with dpar[0] = 1e-12 on SQUARED
# residual norms and x0 = 0 (blascoCodinaHuerta.cpp:3998-4018), i.e.
# ||r||_2 <= 1e-6 ||b||_2 on the plain 2-norm.
REF_CG_RTOL = 1e-6
REF_CG_MAXIT = 1000

# Nodes stored in full up to this count; larger meshes store a strided
# sample plus whole-field norms and weighted checksums.
FULL_NODES = 6000


def perturbed_box(nx, ny, nz, amp, seed):
    """Corner nodes of an nx x ny x nz box with interior nodes moved by a
    seeded random offset (non-affine elements exercise the full Jacobian),
    the connectivity and the velocity-BC faces (lid = BC 2, listed last)."""
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


# name -> what the deck exercises
CASES = {
    "c1": "8^3 cavity, Re 100, dt 0.01, 20 steps (the 8^3 benchmark configuration)",
    "c1_runout": "8^3 cavity with maxIter 2: every step ends with its sub-iteration loop run out",
    "graded": "6^3 sinh-graded cavity (grading 1.5), Re 400, dt 0.005, 5 steps",
    "perturbed": "5x4x3 box with randomly moved interior nodes (non-affine elements), 5 steps",
    "duct_small": "3x3x16 bent square duct, plug inlet from the deck, outflow faces, 3 steps",
    "steady": "4^3 cavity, Re 10, converge 0.05: the steady-state test stops the run",
    "c16": "16^3 cavity, Re 400, dt 0.005, 10 steps",
}

# Cases small enough for the GPU parity test's whole-run loop.
GPU_CASES = ("c1", "c1_runout", "graded", "perturbed", "duct_small", "steady", "c16")


def deck_text(name: str) -> str:
    from cfdfs import meshgen
    if name == "c1":
        return meshgen.cavity_deck(meshgen.CavitySpec(8, re=100, dt=0.01, steps=20, ngp=8))
    if name == "c1_runout":
        return meshgen.cavity_deck(meshgen.CavitySpec(8, re=100, dt=0.01, steps=5, ngp=8, max_iter=2))
    if name == "graded":
        return meshgen.cavity_deck(meshgen.CavitySpec(6, re=400, dt=0.005, steps=5, ngp=8, grading=1.5))
    if name == "perturbed":
        xyz, conn, faces = perturbed_box(5, 4, 3, 0.2, seed=7)
        return meshgen.deck_from_arrays(xyz, conn, faces, [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0)], zero_p_node1=3,
                                        ngp=8, dt=0.01, steps=5, viscosity=0.01)
    if name == "duct_small":
        return meshgen.duct_deck(n_cross=3, n_axial=16, steps=3, dt=0.01)
    if name == "steady":
        return meshgen.cavity_deck(meshgen.CavitySpec(4, re=10, dt=0.01, steps=100, ngp=8, converge=0.05))
    if name == "c16":
        return meshgen.cavity_deck(meshgen.CavitySpec(16, re=400, dt=0.005, steps=10, ngp=8))
    raise KeyError(name)


def write_deck(name: str, path: str) -> str:
    text = deck_text(name)
    with open(path, "w") as f:
        f.write(text)
    return path


def sha256_text(text: str) -> str:
    return hashlib.sha256(text.encode()).hexdigest()


# The shipped 30^3 graded cavity deck of the reference
# (inputFiles/lidDrivenCavity/lidDrivenCavity_NE27000.inp), cut to 3 time
# steps by its t_final line.  It is not part of this repository; tests that
# need it look for it under $CFD_REFERENCE_DIR and skip without it.
SHIPPED_REL = os.path.join("inputFiles", "lidDrivenCavity", "lidDrivenCavity_NE27000.inp")
SHIPPED_STEPS = 3


def shipped_deck_path() -> str | None:
    base = os.environ.get("CFD_REFERENCE_DIR", "")
    p = os.path.join(base, SHIPPED_REL) if base else ""
    return p if p and os.path.exists(p) else None


def shipped_deck_text(src: str, steps: int = SHIPPED_STEPS) -> str:
    """The shipped deck with t_final set so that the reference's
    while (timeT < t_final) loop runs ``steps`` steps of its dt (1e-3)."""
    out = []
    for line in open(src).read().split("\n"):
        if line.startswith("t_final"):
            line = "t_final  : %r" % ((steps - 0.5) * 1e-3)
        out.append(line)
    return "\n".join(out)


# ---------------------------------------------------------------- readers

def parse_dat(text: str) -> dict:
    """Reads a createTecplot file: the title, the node rows (x y z u v w p,
    in the solver's node numbering) and the sub-brick connectivity rows.
    Hashes of the coordinate text and of the connectivity text identify the
    node numbering and element-to-node map exactly."""
    lines = text.split("\n")
    zone = lines[2]
    nn = int(re.search(r"N=(\d+)", zone).group(1))
    ne8 = int(re.search(r"E=(\d+)", zone).group(1))
    rows = lines[3:3 + nn]
    toks = [r.split() for r in rows]
    xyz_text = "\n".join(" ".join(t[:3]) for t in toks)
    vals = np.array([[float(v) for v in t[3:7]] for t in toks])
    conn = "\n".join(l.strip() for l in lines[3 + nn:3 + nn + ne8])
    return dict(title=lines[0], variables=lines[1], zone=zone, nn=nn, ne8=ne8,
                xyz_sha=sha256_text(xyz_text), conn_sha=sha256_text(conn), uvwp=vals.T.copy())


_MON = re.compile(r"^\s*(\d+)\s+(\d+)\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)"
                  r"\s+(-?\d+\.\d+)\s+(-?\d+\.\d+)\s*$")
_CG = re.compile(r"MKL_CG converged after (\d+) iterations\.")


def parse_stdout(text: str):
    """CG iterations of every pressure solve and the monitor rows of the
    reference's screen output.  A monitor row is
    "%6d  %6d  %10.5f  %12.5f  %12.5f  %12.5f  %12.5f %12.5f %12.5f" with
    (timeN, iter, timeT, u, v, w, p, step wall time, maxAcc); the returned
    rows drop the wall time, and ``mon_text`` holds each row's text with the
    wall-time field removed."""
    cg, mon, mon_text = [], [], []
    for line in text.split("\n"):
        m = _CG.search(line)
        if m:
            cg.append(int(m.group(1)))
            continue
        m = _MON.match(line)
        if m:
            g = m.groups()
            mon.append([float(g[i]) for i in (0, 1, 2, 3, 4, 5, 6, 8)])
            mon_text.append(monitor_text(*[float(g[i]) for i in (0, 1, 2, 3, 4, 5, 6, 8)]))
    return np.array(cg, dtype=np.int32), np.array(mon).reshape(-1, 8), mon_text


def monitor_text(step, it, t, u, v, w, p, max_acc) -> str:
    """One monitor row in the reference's format without its wall-time field."""
    return "%6d  %6d  %10.5f  %12.5f  %12.5f  %12.5f  %12.5f %12.5f" % (int(step), int(it), t, u, v, w, p,
                                                                         max_acc)


# ------------------------------------------------------------ summaries

def field_weights(n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.float64)
    return np.sin(0.7 * i + 0.3) * (1.0 + 0.5 * np.cos(0.013 * i))


def summarize(uvwp: np.ndarray) -> dict:
    """What a fixture keeps of the 4 x NN final fields (u, v, w, p on every
    velocity node, p interpolated on the non-corner nodes as createTecplot
    does): the sample rows, whole-field 2-norms and weighted checksums."""
    nn = uvwp.shape[1]
    idx = np.arange(nn) if nn <= FULL_NODES else np.arange(0, nn, max(1, nn // FULL_NODES))
    w = field_weights(nn)
    return dict(idx=idx.astype(np.int64), sample=uvwp[:, idx].copy(), norms=np.linalg.norm(uvwp, axis=1),
                wsum=(uvwp * w).sum(axis=1), asum=np.abs(uvwp * w).sum(axis=1))


def compare_summary(fix, uvwp: np.ndarray) -> dict:
    """Relative differences of a run's final fields against a fixture, per
    field (u, v, w, p): sample rel. L2, norm, weighted checksum."""
    s = summarize(uvwp)
    out = {}
    for k, name in enumerate("uvwp"):
        a, b = s["sample"][k], fix["sample"][k]
        nb = np.linalg.norm(b)
        out[name] = dict(
            sample=float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)),
            norm=float(abs(s["norms"][k] - fix["norms"][k]) / max(fix["norms"][k], 1e-300)),
            wsum=float(abs(s["wsum"][k] - fix["wsum"][k]) / max(fix["asum"][k], 1e-300)))
    return out


def load_fixture(name: str, golden_dir: str) -> dict:
    with np.load(os.path.join(golden_dir, f"ref_{name}.npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}
