"""Input-deck generators in the fractional-step ``.inp`` format.

The format is the one read by ``readInputFile``
(fractionalStep/Cpp/blascoCodinaHuerta.cpp:528-725): two title lines, eighteen
``key : value`` header lines, then corner-node coordinates, hex8 corner
connectivity, the BC table, the velocity-BC and outflow face lists, the node
where pressure is pinned and the monitor-point coordinates.  Ids in the file
are 1-based.  The layout of the shipped deck
inputFiles/lidDrivenCavity/lidDrivenCavity_NE27000.inp is followed:

* corner nodes numbered lexicographically with x fastest;
* element corners c1 (0,0,0), c2 +x, c3 +x+y, c4 +y, c5..c8 the same at +z;
* velocity-BC faces listed bottom (face 1), x=0 (face 5), x=1 (face 3),
  y=0 (face 2), y=1 (face 4) and the lid (face 6) last, so that the lid
  value wins on the lid edges (later faces overwrite earlier ones);
* pressure pinned at the centre of the bottom face, monitor at the centre.

Generators for the cavity (uniform or sinh-graded) and for the bent square
duct live here; the reference's own MATLAB generators write an older format.
"""
from __future__ import annotations

import io
import math
import os

import numpy as np

__all__ = ["CavitySpec", "cavity_arrays", "cavity_deck", "write_cavity", "steps_for", "duct_arrays", "duct_deck",
           "write_duct", "t_final_for_steps", "deck_from_arrays", "write_text"]


def steps_for(dt: float, t_final: float, t_ini: float = 0.0) -> int:
    """Number of steps the reference's ``while (timeT < t_final) timeT += dt``
    loop runs, evaluated in the same FP64 arithmetic
    (blascoCodinaHuerta.cpp:2859-2862)."""
    t, n = t_ini, 0
    while t < t_final:
        t = t + dt
        n += 1
    return n


def t_final_for_steps(dt: float, steps: int) -> float:
    """A ``t_final`` for which the reference loop runs exactly ``steps`` steps:
    ``steps*dt`` when FP64 accumulation agrees, else ``(steps-0.5)*dt``."""
    tf = steps * dt
    if steps_for(dt, tf) == steps:
        return tf
    tf = (steps - 0.5) * dt
    assert steps_for(dt, tf) == steps
    return tf


def _grid_1d(n: int, grading: float) -> np.ndarray:
    """Node positions on [0, 1]; grading > 0 clusters nodes towards both ends
    with a sinh map (the clustering used by the reference's cavity mesh
    generator, oldFiles/meshGenerators&Converters/cavityMeshGenerator.m:46-60,
    written here from the formula x = 0.5*(1 + sinh(g*(2s-1))/sinh(g)))."""
    s = np.linspace(0.0, 1.0, n + 1)
    if grading <= 0.0:
        return s
    x = 0.5 * (1.0 + np.sinh(grading * (2.0 * s - 1.0)) / math.sinh(grading))
    x[0], x[-1] = 0.0, 1.0
    return x


def _fmt_header(title: str, ne: int, ncn: int, ngp: int, dt: float, t_final: float, max_iter: int,
                tol: float, converge: float, density: float, viscosity: float) -> str:
    sep = "=" * 48
    lines = [
        title,
        sep,
        f"eType    : 1",
        f"NE       : {ne}",
        f"NCN      : {ncn}",
        f"NENv     : 27",
        f"NENp     : 8",
        f"NGP      : {ngp}",
        f"alpha    : 1.000000",
        f"dt       : {dt!r}",
        f"t_ini    : 0.000000",
        f"t_final  : {t_final!r}",
        f"maxIter  : {max_iter}",
        f"tolerance: {tol!r}",
        f"converge : {converge!r}",
        f"isRestart: 0",
        f"density  : {density!r}",
        f"viscosity: {viscosity!r}",
        f"fx       : 0.0",
        f"fy       : 0.0",
        sep,
    ]
    return "\n".join(lines) + "\n"


def _write_body(buf: io.StringIO, xyz: np.ndarray, conn: np.ndarray, bcs, vel_faces: np.ndarray,
                out_faces: np.ndarray, zero_p_node1: int, monitor) -> None:
    sep = "=" * 48
    buf.write("Corner Node No         x                y                z\n")
    ids = np.arange(1, xyz.shape[0] + 1)
    buf.write("".join(f"{i:9d}   {x:16.9f} {y:16.9f} {z:16.9f}\n" for i, (x, y, z) in zip(ids, xyz.tolist())))
    buf.write(sep + "\n")
    buf.write("Elem No   corner1  corner2  corner3  corner4  corner5  corner6  corner7  corner8\n")
    eids = np.arange(1, conn.shape[0] + 1)
    buf.write("".join(f"{e:6d} " + " ".join(f"{c:8d}" for c in row) + " \n"
                      for e, row in zip(eids.tolist(), (conn + 1).tolist())))
    buf.write(sep + "\n")
    buf.write("BCs (Number of specified BCs, their types and strings) \n")
    buf.write(f"nBC       : {len(bcs)} \n")
    for k, (u, v, w) in enumerate(bcs):
        buf.write(f"BC {k + 1}      : 1  {u!r} : {v!r} : {w!r}\n")
    buf.write(sep + "\n")
    buf.write(f"nVelFaces : {vel_faces.shape[0]} \n")
    buf.write(f"nOutFaces : {out_faces.shape[0]} \n")
    buf.write(sep + "\n")
    buf.write("Velocity BC (Elem# Face# BC#)\n")
    buf.write("".join(f"{e:5d}{f:5d}{b:5d}\n" for e, f, b in vel_faces.tolist()))
    buf.write(sep + "\n")
    buf.write("Outflow BC (Elem# Face# BC#)\n")
    buf.write("".join(f"{e:5d}{f:5d}{b:5d}\n" for e, f, b in out_faces.tolist()))
    buf.write(sep + "\n")
    buf.write("Node number where pressure is taken to be zero\n")
    buf.write(f"{zero_p_node1}\n")
    buf.write(sep + "\n")
    buf.write("Monitor point coordinates\n")
    buf.write(f"{monitor[0]!r}  {monitor[1]!r}  {monitor[2]!r}\n")


class CavitySpec:
    """Parameters of a structured lid-driven cavity on the unit cube."""

    def __init__(self, n: int, re: float = 100.0, dt: float = 0.01, steps: int = 20, ngp: int = 8,
                 lid: float = 1.0, max_iter: int = 4, tol: float = 1e-3, converge: float = 1e-6,
                 grading: float = 0.0, density: float = 1.0):
        self.n, self.re, self.dt, self.steps, self.ngp = n, re, dt, steps, ngp
        self.lid, self.max_iter, self.tol, self.converge = lid, max_iter, tol, converge
        self.grading, self.density = grading, density


def cavity_arrays(n: int, grading: float = 0.0):
    """Corner coordinates (NCN x 3), connectivity (NE x 8, 0-based) and the
    velocity-BC face list (elem 1-based, face 1-based, bc 1-based)."""
    g = _grid_1d(n, grading)
    m = n + 1
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    xyz = np.stack([g[i.ravel()], g[j.ravel()], g[k.ravel()]], axis=1)
    ek, ej, ei = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ei, ej, ek = ei.ravel(), ej.ravel(), ek.ravel()
    node = lambda a, b, c: a + m * b + m * m * c
    conn = np.stack([node(ei, ej, ek), node(ei + 1, ej, ek), node(ei + 1, ej + 1, ek), node(ei, ej + 1, ek),
                     node(ei, ej, ek + 1), node(ei + 1, ej, ek + 1), node(ei + 1, ej + 1, ek + 1),
                     node(ei, ej + 1, ek + 1)], axis=1).astype(np.int64)
    eid = np.arange(n ** 3) + 1
    faces = []
    for face, sel, bc in ((1, ek == 0, 1), (5, ei == 0, 1), (3, ei == n - 1, 1), (2, ej == 0, 1),
                          (4, ej == n - 1, 1), (6, ek == n - 1, 2)):
        e = eid[sel]
        faces.append(np.stack([e, np.full_like(e, face), np.full_like(e, bc)], axis=1))
    return xyz, conn, np.concatenate(faces, axis=0)


def cavity_deck(spec: CavitySpec) -> str:
    """The ``.inp`` text of a lid-driven cavity: no-slip on five faces (BC 1),
    lid velocity (lid, 0, 0) on z = 1 (BC 2, listed last)."""
    n = spec.n
    xyz, conn, vel_faces = cavity_arrays(n, spec.grading)
    t_final = t_final_for_steps(spec.dt, spec.steps)
    half = n // 2
    zero_p = 1 + half + half * (n + 1)  # bottom-face centre, 1-based
    buf = io.StringIO()
    buf.write(_fmt_header(f"3D Lid-driven cavity {n}x{n}x{n}, Re={spec.re:g}", n ** 3, (n + 1) ** 3,
                          spec.ngp, spec.dt, t_final, spec.max_iter, spec.tol, spec.converge, spec.density,
                          spec.lid / spec.re))
    _write_body(buf, xyz, conn, [(0.0, 0.0, 0.0), (float(spec.lid), 0.0, 0.0)], vel_faces,
                np.zeros((0, 3), dtype=np.int64), zero_p, (0.5, 0.5, 0.5))
    return buf.getvalue()


def deck_from_arrays(xyz, conn, vel_faces, bcs, *, out_faces=None, zero_p_node1=2, monitor=(0.5, 0.5, 0.5),
                     ngp=8, dt=0.01, steps=10, max_iter=4, tol=1e-3, converge=1e-6, density=1.0,
                     viscosity=0.01, title="generated deck") -> str:
    """``.inp`` text from arrays: corner coordinates (NCN x 3), 0-based
    connectivity (NE x 8), velocity faces (rows of 1-based element, face,
    bc), BC values [(u, v, w), ...]."""
    xyz = np.asarray(xyz, dtype=np.float64)
    conn = np.asarray(conn, dtype=np.int64)
    vel_faces = np.asarray(vel_faces, dtype=np.int64).reshape(-1, 3)
    out_faces = np.zeros((0, 3), dtype=np.int64) if out_faces is None else np.asarray(out_faces).reshape(-1, 3)
    buf = io.StringIO()
    buf.write(_fmt_header(title, conn.shape[0], xyz.shape[0], ngp, dt, t_final_for_steps(dt, steps), max_iter, tol,
                          converge, density, viscosity))
    _write_body(buf, xyz, conn, bcs, vel_faces, out_faces, zero_p_node1, monitor)
    return buf.getvalue()


def write_text(path: str, text: str) -> str:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)
    return path


def write_cavity(path: str, spec: CavitySpec) -> str:
    text = cavity_deck(spec)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)
    return path


# ---------------------------------------------------------------------------
# Bent square duct: straight inlet leg, 90-degree bend, straight outlet leg.
# ---------------------------------------------------------------------------

def duct_arrays(n_cross: int = 24, n_axial: int = 160, leg: float = 3.0, radius: float = 2.0,
                side: float = 1.0):
    """Body-fitted hex mesh of a square duct of side ``side`` whose centreline
    runs along +x for ``leg``, turns 90 degrees about the z axis with
    centreline radius ``radius`` (towards +y), then runs along +y for ``leg``.

    Axial elements are distributed proportionally to the centreline length of
    each part.  Returns corner coordinates, connectivity (0-based), and the
    inlet / wall / outlet element faces (element 1-based, face 1-based)."""
    arc = 0.5 * math.pi * radius
    total = 2 * leg + arc
    n1 = max(1, round(n_axial * leg / total))
    n3 = n1
    n2 = n_axial - n1 - n3
    # centreline parameter s_k and local frame for every axial station
    stations = []
    for k in range(n_axial + 1):
        if k <= n1:
            t = leg * k / n1
            c = np.array([t, 0.0, 0.0]); tang = np.array([1.0, 0.0, 0.0])
        elif k <= n1 + n2:
            th = 0.5 * math.pi * (k - n1) / n2
            c = np.array([leg + radius * math.sin(th), radius * (1 - math.cos(th)), 0.0])
            tang = np.array([math.cos(th), math.sin(th), 0.0])
        else:
            t = leg * (k - n1 - n2) / n3
            c = np.array([leg + radius, radius + t, 0.0]); tang = np.array([0.0, 1.0, 0.0])
        normal = np.array([-tang[1], tang[0], 0.0])  # in-plane normal (towards bend centre)
        stations.append((c, normal))
    m = n_cross + 1
    a = np.linspace(-0.5 * side, 0.5 * side, m)
    # node (i: axial, j: across in-plane, l: across z); x fastest = axial index
    xyz = np.empty(((n_axial + 1) * m * m, 3))
    idx = 0
    for l in range(m):
        for j in range(m):
            for k in range(n_axial + 1):
                c, nrm = stations[k]
                p = c + a[j] * nrm + np.array([0.0, 0.0, a[l]])
                xyz[idx] = p
                idx += 1
    na = n_axial + 1
    node = lambda k, j, l: k + na * j + na * m * l
    conn, eid = [], 0
    inlet, outlet, walls = [], [], []
    for l in range(n_cross):
        for j in range(n_cross):
            for k in range(n_axial):
                conn.append([node(k, j, l), node(k + 1, j, l), node(k + 1, j + 1, l), node(k, j + 1, l),
                             node(k, j, l + 1), node(k + 1, j, l + 1), node(k + 1, j + 1, l + 1),
                             node(k, j + 1, l + 1)])
                eid += 1
                if k == 0:
                    inlet.append((eid, 5))
                if k == n_axial - 1:
                    outlet.append((eid, 3))
                if l == 0:
                    walls.append((eid, 1))
                if l == n_cross - 1:
                    walls.append((eid, 6))
                if j == 0:
                    walls.append((eid, 2))
                if j == n_cross - 1:
                    walls.append((eid, 4))
    return xyz, np.asarray(conn, dtype=np.int64), inlet, walls, outlet


def duct_deck(n_cross: int = 24, n_axial: int = 160, re: float = 200.0, dt: float = 0.005,
              steps: int = 300, ngp: int = 8, max_iter: int = 4, tol: float = 1e-3,
              converge: float = 1e-6) -> str:
    """``.inp`` text of the bent square duct.  BC 1 = inlet (1, 0, 0) (the
    uniform part of the profile; a per-node parabolic profile is supplied
    separately because the deck holds one constant value per BC id), BC 2 =
    no-slip walls listed after the inlet so walls own the inlet rim; outlet
    faces are listed as outflow (natural, zero traction).  Viscosity = 1/Re
    with the duct side and the inlet peak speed as scales."""
    xyz, conn, inlet, walls, outlet = duct_arrays(n_cross, n_axial)
    vel = np.array([(e, f, 1) for e, f in inlet] + [(e, f, 2) for e, f in walls], dtype=np.int64)
    outf = np.array([(e, f, 1) for e, f in outlet], dtype=np.int64).reshape(-1, 3)
    t_final = t_final_for_steps(dt, steps)
    ne = conn.shape[0]
    # pressure pinned at an outlet corner node with 1-based id >= 2
    last_face_nodes = conn[[e - 1 for e, _ in outlet]][:, [1, 2, 5, 6]].ravel()
    zero_p = int(np.max(last_face_nodes)) + 1
    buf = io.StringIO()
    buf.write(_fmt_header(f"Bending square duct {n_cross}x{n_cross}x{n_axial}, Re={re:g}", ne, xyz.shape[0], ngp,
                          dt, t_final, max_iter, tol, converge, 1.0, 1.0 / re))
    mid = xyz.mean(axis=0)
    _write_body(buf, xyz, conn, [(1.0, 0.0, 0.0), (0.0, 0.0, 0.0)], vel, outf, zero_p, tuple(mid.tolist()))
    return buf.getvalue()


def duct_inlet_profile(mesh, peak: float = 1.0, side: float = 1.0):
    """Per-node parabolic inlet velocity of a duct deck: the nodes that keep
    BC 1 (0-based id 0 in ``HostMesh.bcnodes``; wall nodes on the inlet rim
    belong to BC 2) get
    u = peak (1 - (2y/side)^2) (1 - (2z/side)^2) along +x, v = w = 0.
    ``mesh`` is a ``cfdfs.HostMesh`` of the deck.  Returns (nodes, uvw) for
    ``Solver.set_bc_values``."""
    bc = mesh.bcnodes()
    xyz = mesh.coord()
    nodes = bc[bc[:, 1] == 0, 0].astype(np.int32)
    y, z = xyz[nodes, 1] / (0.5 * side), xyz[nodes, 2] / (0.5 * side)
    u = peak * np.clip(1.0 - y * y, 0.0, None) * np.clip(1.0 - z * z, 0.0, None)
    uvw = np.zeros((len(nodes), 3))
    uvw[:, 0] = u
    return nodes, uvw


def duct_grid_dims(n_cross: int = 24, n_axial: int = 160):
    """Pressure-node grid (nx, ny, nz) of ``duct_arrays``: corner nodes are
    numbered axial index fastest, then across in-plane, then across z."""
    return (n_axial + 1, n_cross + 1, n_cross + 1)


def write_duct(path: str, **kw) -> str:
    text = duct_deck(**kw)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)
    return path
