"""The bench's bookkeeping on the CPU: bench.run_ours driven by a stand-in
solver whose every timed region takes 100 ms (tests/bench_fake_run.py, in
its own process) prints one JSON line with the keys the bench contract
needs and the arithmetic those times imply."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_bench_line_from_stand_in_solver():
    r = subprocess.run([sys.executable, os.path.join(HERE, "bench_fake_run.py")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "step_roofline", "e2e",
                "gpu_launches", "clocks", "pressure_fallbacks", "fp64_path", "twolevel_path", "accuracy"):
        assert key in line, key
    # 4 timed steps in 100 ms on one replica
    assert line["value"] == pytest.approx(40.0) and line["ms_per_step"] == pytest.approx(25.0)
    assert line["config"]["workload"].startswith("lid-driven cavity")
    assert line["e2e"]["h2d_bytes_per_step"] == line["e2e"]["d2h_bytes_per_step"] > 0
    sr = line["step_roofline"]
    # achieved is printed to 0.1 GB/s
    assert sr["bytes_per_step"] > 0 and abs(sr["frac"] * sr["peak"] - sr["achieved"]) <= 0.05 + 1e-3 * sr["achieved"]
    assert line["e2e"]["steps"] == line["steps"]
    assert line["roofline"]["kernel"] == "spmv_z"


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "fs_ref")),
                    reason="the reference program was not built on this machine")
def test_reference_arm_runs_the_reference_program():
    """bench.py --impl reference on a 4^3 cavity: the reference's own program
    (oracle/_ref/fs_ref) timed by its own TimeSpend column, one JSON line in
    the contract's form."""
    root = os.path.dirname(HERE)
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--n", "4",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "steps/s" and line["value"] > 0
    assert line["steps"] == 3 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
