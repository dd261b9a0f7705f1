"""Golden end states of whole runs at full configuration size, made by the CPU
oracle (oracle/fs_oracle.cpp, FP64, Jacobi-PCG rtol 1e-8, x0 = 0).

A full run of the oracle at these sizes takes minutes on the host cores, which
is too long to repeat in every GPU test run.  This script runs it once and
stores a strided subsample of the final velocity and pressure, the norms of
the whole fields and the run counters.  The GPU tests compare their own full
runs with these files.

Cases:
- ``c2_cavity32``: lid-driven cavity, 32^3 hex27/hex8 elements, Re 400,
  dt 0.005, 200 steps, NGP 8 (the FP64 drop-in configuration).
- ``c3_cavity64``: lid-driven cavity, 64^3 elements, Re 1000, dt 0.002,
  100 steps, NGP 8 (the configuration of the headline benchmark).
- ``duct_24x160``: bent square duct (inlet leg 3, 90-degree bend of
  centreline radius 2, outlet leg 3), 24 x 24 elements across by 160 along,
  Re 200, dt 0.005, 300 steps, NGP 8, parabolic inlet of peak 1.0 set on the
  inlet nodes after step0 (``meshgen.duct_inlet_profile``), no-slip walls,
  natural outlet.

Usage (from the repository root): ``python tests/golden/make_run_goldens.py``
"""
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cfd-with-cuda_b200"))

# strides of the stored subsamples: every u_stride-th entry of [u | v | w]
# and every p_stride-th pressure node (about 60 KB per file)
CASES = {
    "c2_cavity32": dict(kind="cavity", n=32, re=400.0, dt=0.005, steps=200, ngp=8, u_stride=163, p_stride=13),
    "duct_24x160": dict(kind="duct", n_cross=24, n_axial=160, re=200.0, dt=0.005, steps=300, ngp=8,
                        u_stride=499, p_stride=37),
    "c3_cavity64": dict(kind="cavity", n=64, re=1000.0, dt=0.002, steps=100, ngp=8, u_stride=1499,
                        p_stride=101),
}


def deck_for(case: str, directory: str) -> str:
    from cfdfs import meshgen
    c = CASES[case]
    path = os.path.join(directory, f"{case}.inp")
    if c["kind"] == "duct":
        return meshgen.write_duct(path, n_cross=c["n_cross"], n_axial=c["n_axial"], re=c["re"], dt=c["dt"],
                                  steps=c["steps"], ngp=c["ngp"])
    return meshgen.write_cavity(path, meshgen.CavitySpec(c["n"], re=c["re"], dt=c["dt"], steps=c["steps"],
                                                         ngp=c["ngp"]))


def inlet_for(case: str, mesh):
    """(nodes, uvw) of the duct's parabolic inlet, or None; ``mesh`` has
    ``bcnodes()`` and ``coord()`` (the oracle or ``cfdfs.HostMesh``)."""
    from cfdfs import meshgen
    return meshgen.duct_inlet_profile(mesh) if CASES[case]["kind"] == "duct" else None


def make(case: str, out_dir: str) -> str:
    import pyoracle
    pyoracle.build()
    d = tempfile.mkdtemp()
    deck = deck_for(case, d)
    o = pyoracle.Oracle(deck)
    o.step0()
    inlet = inlet_for(case, o)
    if inlet is not None:
        nodes, uvw = inlet
        U = o.vec("Un")
        for k in range(3):
            U[k * o.NN + nodes] = uvw[:, k]
        o.set_vec("Un", U)
    t0 = time.time()
    info = o.run(-1)
    secs = time.time() - t0
    U, P = o.vec("Un"), o.vec("Pn")
    mon = o.mon
    us, ps = CASES[case]["u_stride"], CASES[case]["p_stride"]
    path = os.path.join(out_dir, f"{case}.npz")
    np.savez_compressed(
        path, u_sub=U[::us], p_sub=P[::ps], u_norm=np.linalg.norm(U), p_norm=np.linalg.norm(P),
        u_sum=U.sum(), p_sum=P.sum(), mon=np.array([U[mon], U[o.NN + mon], U[2 * o.NN + mon], P[mon]]),
        steps=info["steps"], subits=info["subits"], cg_its=info["cg_its"], steady=int(info["steady"]),
        max_acc=info["max_acc"], u_stride=us, p_stride=ps, oracle_threads=pyoracle.threads(),
        oracle_seconds=secs)
    o.close()
    return path


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    for name in (sys.argv[1:] or list(CASES)):
        print(make(name, here))
