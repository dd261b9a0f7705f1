"""The committed network, cfd-with-cuda_b200/weights/unet_cavity.bin, and its
training record unet_cavity.json, on the CPU:

- the file is in the library's format: the 8-byte tag "CFDUNET1", an int64
  parameter count, then the FP32 parameters;
- the count matches the library's and the oracle's layout, and every
  parameter is finite;
- the oracle's forward pass of the network on a 17^3 residual is finite and
  not trivial;
- the record states the training command, and its measured quality shows
  the trained correction leaving less Z-norm error than the two-level step
  after 5 and 20 iterations, with no Jacobi-PCG fallback in its
  evaluation runs."""
import json
import os

import numpy as np

import unet_oracle as U

WDIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cfd-with-cuda_b200", "weights")


def _read(path):
    with open(path, "rb") as f:
        tag = f.read(8)
        n = int(np.frombuffer(f.read(8), dtype="<i8")[0])
        theta = np.frombuffer(f.read(), dtype="<f4")
    return tag, n, theta


def test_weight_file_format_and_layout():
    import cfdfs
    tag, n, theta = _read(os.path.join(WDIR, "unet_cavity.bin"))
    assert tag == b"CFDUNET1"
    assert n == U.param_count() == cfdfs.UNet.param_count()
    assert theta.size == n
    assert np.all(np.isfinite(theta))


def test_committed_network_forward_on_the_oracle():
    _, _, theta = _read(os.path.join(WDIR, "unet_cavity.bin"))
    x = np.random.default_rng(11).standard_normal((17, 17, 17)).astype(np.float32)
    x /= np.sqrt(np.mean(x * x))
    out, _ = U.forward(theta, x)
    assert out.shape == x.shape
    assert np.all(np.isfinite(out))
    assert np.std(out) > 1e-3


def test_training_record():
    with open(os.path.join(WDIR, "unet_cavity.json")) as f:
        rec = json.load(f)
    assert "cfdfs.learned" in rec["command"]
    # the configured training set: at least 2000 pairs from seeded cavity
    # runs and the bent duct, before the on-policy pairs
    assert rec["cavity_pairs"] > 0 and rec["duct_pairs"] > 0 and rec["onpolicy_pairs"] > 0
    assert rec["cavity_pairs"] + rec["duct_pairs"] >= 2000
    assert rec["val_loss"] < rec["val_loss_init"]
    q = {e["k"]: e for e in rec["energy_quality"]}
    for k in (0, 5, 20):
        assert q[k]["learned"] < q[k]["twolevel"]
    # held-out evaluation: fewer iterations per solve than two-level CG in
    # every case; a Jacobi-PCG fallback (a stalled flexible-CG solve) in at
    # most one solve of a case
    ev = rec["eval"]
    for case in ("c3_re1000", "seed10000"):
        for prec in ("fp64", "mixed"):
            learned, twolevel = ev[f"{case}_{prec}_learned"], ev[f"{case}_{prec}_twolevel"]
            assert learned["its_per_solve"] < twolevel["its_per_solve"]
            assert learned["fallbacks"] <= 1 and twolevel["fallbacks"] == 0
