"""Generates the reference-parity fixtures ``tests/golden/ref_<case>.npz``.

Runs the reference's own CPU solver -- fractionalStep/Cpp/
blascoCodinaHuerta.cpp, compiled unmodified by ``make -C oracle ref`` against
the stand-in MKL and CSparse of ``oracle/refshim`` into ``oracle/_ref/fs_ref``
-- on every case of ``ref_cases.CASES`` (and on the shipped 30^3 deck cut to
3 steps when the reference tree is found), the way its ``main`` expects: a
``ProblemName.txt`` naming ``<case>``, the deck as ``<case>.inp``, results in
``<case>.dat`` and on the screen.  Each fixture stores the deck's sha256, the
Tecplot header, the hashes of the coordinate and connectivity text (the
reference's node numbering and element-to-node map), a summary of the final
u, v, w, p (``ref_cases.summarize``), the CG iterations of every pressure
solve and the monitor rows.

Needs the reference sources, so it runs only where they are; the fixtures
travel with the repository.

    CFD_REFERENCE_DIR=<reference checkout> python tests/golden/make_ref_goldens.py [case ...]
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "cfd-with-cuda_b200"))

import ref_cases  # noqa: E402


def build_ref(reference: str) -> str:
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s", "ref", f"REFERENCE={reference}"],
                   check=True)
    return os.path.join(ROOT, "oracle", "_ref", "fs_ref")


def run_ref(exe: str, name: str, deck: str) -> dict:
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, name + ".inp"), "w") as f:
            f.write(deck)
        with open(os.path.join(d, "ProblemName.txt"), "w") as f:
            f.write(name + "\n")
        t0 = time.time()
        # One thread.  The reference fixes 8 OpenMP threads
        # (blascoCodinaHuerta.cpp:86, 407), and its greedy colouring can give
        # one colour to an element and its first neighbour (after a conflict
        # it sets i = 0 and the loop's i++ skips neighbour 0,
        # blascoCodinaHuerta.cpp:880-886); its coloured convection loop
        # (blascoCodinaHuerta.cpp:3554-3660) then races on the shared nodes
        # and the result changes from run to run (the 5x4x3 box and the duct
        # of these cases).  OMP_THREAD_LIMIT=1 caps the team whatever
        # omp_set_num_threads asks, which gives the race-free sum in colour
        # order.
        p = subprocess.run([exe], cwd=d, capture_output=True, text=True, check=True,
                           env=dict(os.environ, OMP_THREAD_LIMIT="1"))
        secs = time.time() - t0
        dat = ref_cases.parse_dat(open(os.path.join(d, name + ".dat")).read())
    cg, mon, mon_text = ref_cases.parse_stdout(p.stdout)
    s = ref_cases.summarize(dat["uvwp"])
    return dict(deck_sha256=np.array(ref_cases.sha256_text(deck)), title=np.array(dat["title"]),
                variables=np.array(dat["variables"]), zone=np.array(dat["zone"]),
                xyz_sha=np.array(dat["xyz_sha"]), conn_sha=np.array(dat["conn_sha"]),
                cg_iters=cg, mon=mon, mon_text=np.array(mon_text), seconds=np.array(secs), **s)


def main(argv):
    reference = os.environ.get("CFD_REFERENCE_DIR", "")
    if not reference or not os.path.isdir(reference):
        sys.exit("set CFD_REFERENCE_DIR to the reference checkout")
    exe = build_ref(reference)
    names = argv or list(ref_cases.CASES) + ["shipped_ne27000"]
    for name in names:
        if name == "shipped_ne27000":
            src = os.path.join(reference, ref_cases.SHIPPED_REL)
            deck = ref_cases.shipped_deck_text(src)
        else:
            deck = ref_cases.deck_text(name)
        r = run_ref(exe, name, deck)
        out = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(out, **r)
        print(f"{name}: {len(r['mon'])} steps, {len(r['cg_iters'])} solves, {int(r['cg_iters'].sum())} CG its, "
              f"{r['sample'].shape[1]} sampled nodes, {float(r['seconds']):.1f} s -> {os.path.getsize(out)} B")


if __name__ == "__main__":
    main(sys.argv[1:])
