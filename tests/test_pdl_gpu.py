"""Programmatic dependent launch of the two-level iteration's kernels
(CFD_PDL=1): each kernel waits for its predecessor's grid before it reads
anything, so the arithmetic and its order are unchanged and the run must be
bit-identical to the plain launches.  Both runs use the deterministic mode
(coloured convection instead of FP32 atomics), which makes a run
reproducible bit for bit."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(deck, precond, pdl, steps, weights=None):
    import cfdfs
    os.environ["CFD_PDL"] = "1" if pdl else "0"
    try:
        s = cfdfs.Solver(device=0, precision=cfdfs.MIXED, precond=precond, deterministic=1,
                         fcg_net_iters=1 if precond == cfdfs.PC_LEARNED else 0)
    finally:
        del os.environ["CFD_PDL"]
    s.load(deck)
    s.step0()
    if weights:
        s.load_unet(weights)
    st = s.run(steps)
    U, P = s.state()
    s.close()
    return st, U, P


@pytest.mark.parametrize("kind", ["twolevel", "learned"])
def test_pdl_is_bit_identical(kind, tmp_path):
    import cfdfs
    from cfdfs import meshgen
    deck = meshgen.write_cavity(str(tmp_path / "c16.inp"), meshgen.CavitySpec(16, re=400, dt=0.005, steps=5))
    precond = cfdfs.PC_LEARNED if kind == "learned" else cfdfs.PC_TWOLEVEL
    w = os.path.join(os.path.dirname(cfdfs.__file__), "..", "weights", "unet_cavity.bin") if kind == "learned" else None
    sa, Ua, Pa = _run(deck, precond, True, 5, w)
    sb, Ub, Pb = _run(deck, precond, False, 5, w)
    assert sa.steps == sb.steps == 5
    assert sa.cg_iters == sb.cg_iters and sa.subiters == sb.subiters
    assert np.array_equal(Ua, Ub) and np.array_equal(Pa, Pb)
