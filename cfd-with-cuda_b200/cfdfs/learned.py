"""Learned pressure preconditioner: training data from the solver's own
pressure solves, and training of the U-Net on the GPU with the library's
forward and backward kernels.

The preconditioner is z = L(r) + f(r / s) s / d: the linear two-level part
L(r) = D^-1 r + P Zc^-1 P^T r (Jacobi step plus the Galerkin coarse-space
correction) and the network's correction f, evaluated on the residual
scaled to unit RMS (s = RMS(r)) and brought back by s / d (d = median
diagonal of Z).  Neither the residual's size nor the mesh spacing reaches
the network, and a network that outputs zero leaves the two-level method.

Data.  For a right-hand side R2 met during a run, a FP64 two-level CG solve
to ||r|| <= 1e-12 ||R2|| gives x*; the same solve stopped after k
iterations gives x_k (x_0 = 0), and flexible CG with the network trained so
far gives the on-policy x_k; each pair is the input x = r_k / s and the
target t = (e_k - L(r_k)) d / s with r_k = R2 - Z x_k, e_k = x* - x_k.
Cavity runs draw Re ~ U[100, 1000] and lid speed ~ U[0.5, 1.5] from
numpy.random.Generator(PCG64(seed)), with dt = 0.002 capped by
``stable_dt`` (the scheme treats convection and viscosity explicitly); duct
runs use the bent duct with a parabolic inlet.

Run ``python -m cfdfs.learned --out weights.bin`` on a GPU machine; it
writes the weights and a JSON log of the data, the loss curve and the
flexible-CG evaluation.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import FP64, MIXED, PC_JACOBI, PC_LEARNED, PC_TWOLEVEL, CfdError, HostMesh, Solver, UNet, meshgen

KS = (0, 2, 5, 10, 20)  # two-level CG iterations of the x_k in each pair
FCG_KS = (1, 2, 4, 8, 16)  # flexible-CG iterations of the on-policy x_k


def cavity_params(seed: int):
    """(Re, lid speed) of a seeded cavity run."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return float(rng.uniform(100.0, 1000.0)), float(rng.uniform(0.5, 1.5))


def stable_dt(dt: float, re: float, lid: float, n: int) -> float:
    """dt capped for the explicit steps of the scheme: the convective number
    lid dt / h_v stays at or below that of the 64^3, lid-1 benchmark case, and
    the diffusion number nu dt / h_v^2 at or below 0.08, where h_v = 1/(2n)
    is the velocity-node spacing and nu = lid / re."""
    nu = lid / re
    hv = 1.0 / (2 * n)
    return min(dt / max(1.0, lid), 0.08 * hv * hv / nu)


class PairSampler:
    """FP64 contexts on one deck: ``run`` advances the flow, ``pair`` solves
    for the pairs with the two-level preconditioner (so the running state is
    never disturbed), ``fcg`` (with a network) gives on-policy iterates."""

    def __init__(self, deck: str, dims, device: int = 0, inlet=None, net=None):
        self.dims = tuple(dims)
        cube = self.dims[0] == self.dims[1] == self.dims[2]
        self.fcg = None
        if net is not None:
            # flexible CG with the network being trained: its own iterates
            # give the on-policy pairs
            self.fcg = Solver(device=device, precision=FP64, cg_rtol=1e-12, precond=PC_LEARNED)
            self.fcg.load(deck)
            self.fcg.step0()
            self.fcg.attach_unet(net, self.dims)
        self.run = Solver(device=device, precision=FP64, precond=PC_TWOLEVEL)
        self.run.load(deck)
        self.run.step0()
        if not cube:
            self.run.set_pressure_grid(self.dims)
        if inlet is not None:
            self.run.set_bc_values(*inlet)
        self.pair = Solver(device=device, precision=FP64, cg_rtol=1e-12, cg_maxit=20000, precond=PC_TWOLEVEL)
        self.pair.load(deck)
        self.pair.step0()
        if not cube:
            self.pair.set_pressure_grid(self.dims)
        rp, col, val = self.pair.matrix("Z")
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        diag = val[col == rows]
        self.dinv = 1.0 / diag
        self.dscale = float(np.median(diag))
        self.n = len(rp) - 1
        assert int(np.prod(self.dims)) == self.n

    def linear(self, r):
        """Linear (two-level) part of the preconditioner applied to r."""
        return self.pair.precond_apply(r)

    def close(self):
        self.run.close()
        self.pair.close()
        if self.fcg is not None:
            self.fcg.close()

    def advance(self, nsteps: int, iters=(1, 2)):
        """Runs nsteps time steps; returns the R2 of the given sub-iterations
        of the last one."""
        if nsteps > 1:
            self.run.run(nsteps - 1)
        got = []
        self.run.time_step(after_step2=lambda it: got.append(self.run.vector("R2")) if it in iters else None)
        return got

    def pairs(self, rhs, ks=KS, onpolicy=False):
        """Normalised (input, target) pairs, float32 arrays shaped (nz, ny, nx).
        x_k comes from two-level CG, or with onpolicy from flexible CG with
        the attached network (k iterations, then one Jacobi-PCG iteration)."""
        out = []
        if not np.any(rhs):
            return out
        self.pair.set_options(cg_rtol=1e-12, cg_maxit=20000)
        xs, st = self.pair.pressure_solve(rhs)
        shape = self.dims[::-1]
        it_solver = self.fcg if onpolicy else self.pair
        for k in ks:
            if k == 0:
                xk = np.zeros(self.n)
            else:
                it_solver.set_options(cg_maxit=k)
                xk, _ = it_solver.pressure_solve(rhs)
            r, nr = self.pair.pressure_residual(rhs, xk)
            if nr == 0.0:
                continue
            s = nr / np.sqrt(self.n)
            x = (r / s).astype(np.float32).reshape(shape)
            t = ((xs - xk - self.linear(r)) * (self.dscale / s)).astype(np.float32).reshape(shape)
            out.append((x, t))
        return out


def cavity_pairs(seeds, n=64, dt=0.002, snap_steps=(1, 5, 15, 35, 70, 100), device=0, tmpdir=None, log=None,
                 net=None, ks=KS):
    """Pairs from seeded cavity runs; returns (x, t) stacked arrays.  With a
    network, the x_k are flexible-CG iterates with that network (on-policy
    pairs: the residuals the preconditioner meets inside its own solves)."""
    xs, ts = [], []
    tmpdir = tmpdir or tempfile.mkdtemp()
    for seed in seeds:
        re, lid = cavity_params(seed)
        dts = stable_dt(dt, re, lid, n)
        deck = meshgen.write_cavity(os.path.join(tmpdir, f"cav_{seed}.inp"),
                                    meshgen.CavitySpec(n, re=re, dt=dts, steps=max(snap_steps), ngp=8, lid=lid))
        ps = PairSampler(deck, (n + 1,) * 3, device=device, net=net)
        done, note = 0, "ok"
        try:
            for stp in snap_steps:
                for rhs in ps.advance(stp - done):
                    for x, t in ps.pairs(rhs, ks=ks, onpolicy=net is not None):
                        xs.append(x)
                        ts.append(t)
                done = stp
        except CfdError as e:  # a run that blows up keeps the pairs it gave
            note = f"stopped after step {done}: {e}"
        ps.close()
        if log is not None:
            log.append(dict(source="cavity-onpolicy" if net is not None else "cavity", seed=seed, re=re, lid=lid,
                            dt=dts, pairs=len(xs), note=note))
    return np.stack(xs), np.stack(ts)


def duct_pairs(n_cross=24, n_axial=160, dt=0.005, snap_steps=(1, 10, 30, 60, 100, 150, 200, 250, 300, 301),
               device=0, tmpdir=None, log=None):
    tmpdir = tmpdir or tempfile.mkdtemp()
    deck = meshgen.write_duct(os.path.join(tmpdir, "duct.inp"), n_cross=n_cross, n_axial=n_axial, dt=dt,
                              steps=max(snap_steps))
    hm = HostMesh(deck)
    inlet = meshgen.duct_inlet_profile(hm)
    hm.close()
    ps = PairSampler(deck, meshgen.duct_grid_dims(n_cross, n_axial), device=device, inlet=inlet)
    xs, ts = [], []
    done = 0
    for stp in snap_steps:
        for rhs in ps.advance(stp - done):
            for x, t in ps.pairs(rhs):
                xs.append(x)
                ts.append(t)
        done = stp
    ps.close()
    if log is not None:
        log.append(dict(source="duct", n_cross=n_cross, n_axial=n_axial, pairs=len(xs)))
    return np.stack(xs), np.stack(ts)


def train(net: UNet, sets, budget_s: float, lr0=1e-3, batch=4, seed=0, log=None):
    """Adam with cosine-decayed learning rate for budget_s seconds over the
    given data sets [(x_dev, t_dev, dims, count)] (torch CUDA tensors hold
    the data; the library reads them through their device addresses).
    Batches alternate between sets in proportion to their sizes."""
    rng = np.random.default_rng(seed)
    sizes = np.array([s[3] for s in sets], dtype=np.float64)
    t0 = time.time()
    step = 0
    curve = []
    while True:
        el = time.time() - t0
        if el >= budget_s:
            break
        lr = lr0 * 0.5 * (1 + np.cos(np.pi * el / budget_s)) + 1e-5
        k = rng.choice(len(sets), p=sizes / sizes.sum())
        x, t, dims, cnt = sets[k]
        i0 = int(rng.integers(0, cnt - batch + 1))
        nv = int(np.prod(dims))
        loss = net.train_batch(x.data_ptr() + 4 * i0 * nv, t.data_ptr() + 4 * i0 * nv, dims, lr, on_device=True,
                               nb=batch)
        step += 1
        if step % 25 == 0:
            curve.append((round(el, 2), step, k, float(loss)))
    if log is not None:
        log["train_curve"] = curve
        log["train_steps"] = step
    return step


def eval_loss(net: UNet, x, t, dims):
    """Mean loss over host pairs (no update)."""
    tot = 0.0
    for i in range(len(x)):
        tot += net.gradient(x[i], t[i], dims)[0]
    return tot / max(1, len(x))


def fcg_eval(net_path: str | None, deck: str, steps: int, precision: int, dims=None, inlet=None, device=0,
             precond=None):
    """Pressure-CG iterations and wall time per step of a run, with the
    learned preconditioner (net_path) or, without a network, the given
    linear preconditioner (default Jacobi-PCG)."""
    pc = PC_LEARNED if net_path else (PC_JACOBI if precond is None else precond)
    s = Solver(device=device, precision=precision, precond=pc)
    s.load(deck)
    s.step0()
    if dims is not None and not (dims[0] == dims[1] == dims[2]):
        s.set_pressure_grid(dims)
    if inlet is not None:
        s.set_bc_values(*inlet)
    if net_path:
        s.load_unet(net_path, dims)
    s.run(1)  # warm-up step
    t0 = time.time()
    st = s.run(steps)
    el = time.time() - t0
    res = dict(steps=st.steps, cg_iters=int(st.cg_iters), subiters=int(st.subiters), fallbacks=int(st.fallbacks),
               its_per_solve=st.cg_iters / max(1, st.subiters), ms_per_step=1e3 * el / max(1, st.steps))
    s.close()
    return res


def energy_quality(ps: PairSampler, net: UNet, rhs, ks=(0, 5, 20)):
    """For pairs from one right-hand side: the relative Z-norm error left by
    the best multiple of the preconditioned residual, min_a ||e - a B(r)||_Z
    / ||e||_Z, for B = Jacobi (D^-1 r), B = two-level (L(r)) and B = the
    learned preconditioner (L(r) + network correction).  Smaller is better;
    0 = exact solve."""
    shape = ps.dims[::-1]
    out = []
    zmul = lambda v: -ps.pair.pressure_residual(np.zeros(ps.n), v)[0]
    ps.pair.set_options(cg_rtol=1e-12, cg_maxit=20000)
    xs, _ = ps.pair.pressure_solve(rhs)
    for k in ks:
        if k == 0:
            xk = np.zeros(ps.n)
        else:
            ps.pair.set_options(cg_maxit=k)
            xk, _ = ps.pair.pressure_solve(rhs)
        r, nr = ps.pair.pressure_residual(rhs, xk)
        e = xs - xk
        s = nr / np.sqrt(ps.n)
        bj = ps.dinv * r
        bt = ps.linear(r)
        y = net.forward((r / s).astype(np.float32).reshape(shape), ps.dims).ravel().astype(np.float64)
        bl = bt + y * (s / ps.dscale)
        ee = float(e @ zmul(e))
        res = {}
        for name, b in (("jacobi", bj), ("twolevel", bt), ("learned", bl)):
            zb = zmul(b)
            a = float(b @ zmul(e)) / float(b @ zb)
            d = e - a * b
            res[name] = float(np.sqrt(max(d @ zmul(d), 0.0) / ee))
        out.append(dict(k=k, **res))
    return out


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", required=True, help="weight file to write (one per variant: <out>.<i>)")
    ap.add_argument("--log", default=None, help="JSON log (default: <out>.json)")
    ap.add_argument("--train-seeds", type=int, default=30)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--budget", type=float, default=300.0, help="training seconds per variant")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--variants", default="1,1", help="loss weights 'w_l2,w_h1;w_l2,w_h1;...'")
    ap.add_argument("--no-duct", action="store_true")
    ap.add_argument("--eval-steps", type=int, default=10)
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--onpolicy-rounds", type=int, default=1,
                    help="rounds of pairs from flexible-CG iterates with the network trained so far")
    ap.add_argument("--onpolicy-seeds", type=int, default=10)
    ap.add_argument("--onpolicy-budget", type=float, default=None, help="training seconds per round (default: budget)")
    a = ap.parse_args(argv)
    log = dict(args=vars(a), data=[])
    t0 = time.time()
    cx, ct = cavity_pairs(range(a.train_seeds), n=a.n, log=log["data"])
    log["cavity_pairs"] = len(cx)
    perm = np.random.default_rng(0).permutation(len(cx))  # batches are contiguous runs of pairs
    cx, ct = cx[perm], ct[perm]
    sets = []
    dims_c = (a.n + 1,) * 3
    # hold out the last 5% of cavity pairs for a validation loss
    nval = max(1, len(cx) // 20)
    vx, vt = cx[-nval:], ct[-nval:]
    sets.append((torch.from_numpy(cx[:-nval]).cuda(), torch.from_numpy(ct[:-nval]).cuda(), dims_c, len(cx) - nval))
    if not a.no_duct:
        dx, dt_ = duct_pairs(log=log["data"])
        log["duct_pairs"] = len(dx)
        perm = np.random.default_rng(1).permutation(len(dx))
        dx, dt_ = dx[perm], dt_[perm]
        sets.append((torch.from_numpy(dx).cuda(), torch.from_numpy(dt_).cuda(), meshgen.duct_grid_dims(), len(dx)))
    log["data_seconds"] = time.time() - t0
    del cx, ct
    # held-out evaluation decks: the 64^3 benchmark cavity (Re 1000, lid 1)
    # and an unseen seed
    tmp = tempfile.mkdtemp()
    decks = {"c3_re1000": meshgen.write_cavity(os.path.join(tmp, "c3.inp"),
                                               meshgen.CavitySpec(a.n, re=1000, dt=0.002, steps=100, ngp=8))}
    re, lid = cavity_params(10_000)
    decks["seed10000"] = meshgen.write_cavity(
        os.path.join(tmp, "h.inp"), meshgen.CavitySpec(a.n, re=re, dt=stable_dt(0.002, re, lid, a.n), steps=100,
                                                       ngp=8, lid=lid))
    ps = PairSampler(decks["c3_re1000"], dims_c)
    rhs_eval = ps.advance(20, iters=(1,))[0]
    log["variants"] = []
    for i, spec in enumerate(a.variants.split(";")):
        w_l2, w_h1 = (float(v) for v in spec.split(","))
        path = f"{a.out}.{i}"
        net = UNet(device=0, seed=1234)
        if a.init:
            net.read(a.init)
        net.set_loss(w_l2, w_h1)
        vl = dict(w_l2=w_l2, w_h1=w_h1, weights=path, val_loss_init=eval_loss(net, vx, vt, dims_c))
        t1 = time.time()
        train(net, sets, a.budget, lr0=a.lr, batch=a.batch, log=vl)
        vsets = list(sets)
        vl["onpolicy"] = []
        for rnd in range(a.onpolicy_rounds):
            # pairs from the network's own flexible-CG solves on fresh seeds,
            # then more training on everything gathered so far
            t2 = time.time()
            seeds = range(1000 * (rnd + 1), 1000 * (rnd + 1) + a.onpolicy_seeds)
            ox, ot = cavity_pairs(seeds, n=a.n, net=net, ks=FCG_KS, log=log["data"])
            perm = np.random.default_rng(2 + rnd).permutation(len(ox))
            vsets.append((torch.from_numpy(ox[perm]).cuda(), torch.from_numpy(ot[perm]).cuda(), dims_c, len(ox)))
            del ox, ot
            rl = dict(round=rnd, pairs=vsets[-1][3], data_seconds=time.time() - t2)
            train(net, vsets, a.onpolicy_budget or a.budget, lr0=0.5 * a.lr, batch=a.batch, seed=1 + rnd, log=rl)
            rl["energy_quality"] = energy_quality(ps, net, rhs_eval)
            vl["onpolicy"].append(rl)
        del vsets
        vl["train_seconds"] = time.time() - t1
        vl["val_loss"] = eval_loss(net, vx, vt, dims_c)
        vl["energy_quality"] = energy_quality(ps, net, rhs_eval)
        net.save(path)
        ev = {}
        for name, deck in decks.items():
            for prec, pname in ((FP64, "fp64"), (MIXED, "mixed")):
                ev[f"{name}_{pname}_learned"] = fcg_eval(path, deck, a.eval_steps, prec, dims_c)
        vl["eval"] = ev
        net.close()
        log["variants"].append(vl)
    ps.close()
    base = {}
    for name, deck in decks.items():
        for prec, pname in ((FP64, "fp64"), (MIXED, "mixed")):
            base[f"{name}_{pname}_jacobi"] = fcg_eval(None, deck, a.eval_steps, prec)
            base[f"{name}_{pname}_twolevel"] = fcg_eval(None, deck, a.eval_steps, prec, precond=PC_TWOLEVEL)
    log["eval_jacobi"] = base
    with open(a.log or a.out + ".json", "w") as f:
        json.dump(log, f, indent=1)
    print(json.dumps(dict(jacobi=base, variants=[{k: v for k, v in vl.items() if k != "train_curve"}
                                                 for vl in log["variants"]]), indent=1))


if __name__ == "__main__":
    main()
