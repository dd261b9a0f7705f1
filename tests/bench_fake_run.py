"""Runs bench.run_ours on the CPU with a stand-in solver and stand-in CUDA
events, and prints its JSON line: the bench's bookkeeping (timing
arithmetic, replica rate, roofline and step-roofline figures, e2e and
accuracy blocks) without a GPU.  Started in its own process by
test_bench_plumbing.py, because it replaces torch.cuda entry points."""
import json
import os
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cfd-with-cuda_b200"))

import numpy as np  # noqa: E402
import torch  # noqa: E402

import cfdfs as real  # noqa: E402


class Info:
    NE, NN, NNp, nnzK, nnzG, nnzZ = 8, 125, 27, 3375, 1331, 729


class Stats:
    def __init__(self, n):
        self.steps, self.subiters, self.cg_iters, self.fallbacks = n, 3 * n, 40 * n, 0
        self.steady, self.maxAcc, self.last_iter = 0, 0.1, 3


class StandInSolver:
    KCLASS = real.Solver.KCLASS

    def __init__(self, **kw):
        self.n = 0
        self.U, self.P = np.ones(3 * Info.NN), np.ones(Info.NNp)

    def load(self, deck): pass
    def step0(self): pass
    def load_unet(self, path): pass
    def precond_apply(self, r): return r
    def refresh(self): return Info()
    def set_state(self, U, P): pass
    def profile(self, on): pass
    def close(self): pass
    def vector(self, name): return np.zeros(Info.NNp)
    def profile_fcg2l(self): return dict(restrict=0.01, coarse=0.02, zphase=0.01, nbwait=0.0, spmv=0.2, dotwait=0.02,
                                         update=0.03)

    def run(self, n):
        self.n += n
        return Stats(n)

    @property
    def stream_ptr(self):
        return 0

    def launch_count(self):
        return 100 * self.n

    def state(self, out=None):
        if out is not None:
            out[0][:] = self.U
            out[1][:] = self.P
            return out
        return self.U.copy(), self.P.copy()

    def profile_read(self):
        d = {k: dict(launches=0, ms=0.0, iters=0) for k in self.KCLASS}
        d["spmv_z"] = dict(launches=10, ms=0.3, iters=9)
        d["fcg"] = dict(launches=20, ms=0.2, iters=9)
        d["unet"] = dict(launches=1, ms=0.27, iters=0)
        return d


class Event:
    def __init__(self, enable_timing=True): pass
    def record(self, stream=None): pass
    def elapsed_time(self, other): return 100.0  # ms


def main():
    fake = types.ModuleType("cfdfs")
    for k in ("MIXED", "FP64", "PC_LEARNED", "PC_TWOLEVEL", "PC_JACOBI"):
        setattr(fake, k, getattr(real, k))
    fake.Solver = StandInSolver
    sys.modules["cfdfs"] = fake
    torch.cuda.set_device = lambda *a, **k: None
    torch.cuda.synchronize = lambda *a, **k: None
    torch.cuda.Event = Event
    torch.cuda.ExternalStream = lambda *a, **k: None
    empty = torch.empty
    torch.empty = lambda *a, pin_memory=False, **k: empty(*a, **k)
    import bench
    bench.make_deck = lambda path, n=4: path

    class Args:
        pass
    a = Args()
    a.steps, a.warmup, a.precision, a.n, a.precond, a.weights = 4, 3, "mixed", 4, "learned", bench.WEIGHTS
    a.net_iters, a.fp64_steps, a.profile_steps, a.cg_maxit, a.cg_warm, a.inner_rtol = 1, 1, 2, 5000, 0, 1e-4
    a.cpu_budget, a.cpu_baseline = 1.0, False
    print(json.dumps(bench.run_ours(a, 0, 1, 0)))


if __name__ == "__main__":
    main()
