#!/usr/bin/env python3
"""Benchmark: time steps per second of the fractional-step solver on the
64^3 lid-driven cavity (hex27 velocity / hex8 pressure, Re 1000, dt 0.002),
the workload the headline metric is quoted on.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  The path does not shard: every
rank runs an independent replica of the same solve ("replicas only"), so the
job value is the sum of the per-rank step rates measured over the slowest
rank's time (weak scaling, no data-path collective).

Timed region: K time steps after W warm-up steps, bracketed by a process
barrier and a device synchronize, measured with CUDA events recorded on the
solver's own stream; the working set (K alone is 1.6 GB FP64) is larger than
the 126 MB L2, so no flush is needed between steps.  Rank 0 prints one JSON
line.  ``--impl reference`` times the reference's own CPU solver
(fractionalStep/Cpp/blascoCodinaHuerta.cpp compiled unmodified into
oracle/_ref/fs_ref against the stand-in MKL and CSparse of oracle/refshim) on
the host cores, with the thread count it sets itself; the C++ restatement
(the oracle) stands in only where that binary was not built.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cfd-with-cuda_b200"))

METRIC = "steps/s at 64³ cavity: mixed+learned-precond vs plain FP64 CG, rel err≤1e-6"
def workload(n):
    return (f"lid-driven cavity {n}x{n}x{n} hex27/hex8 ({2 * n + 1}^3 velocity, {n + 1}^3 pressure nodes), "
            "Re=1000, dt=0.002")
N_ELEM, RE, DT, T_STEPS = 64, 1000.0, 0.002, 100
WEIGHTS = os.path.join(ROOT, "cfd-with-cuda_b200", "weights", "unet_cavity.bin")


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def make_deck(path: str, n: int = N_ELEM) -> str:
    from cfdfs import meshgen
    if not os.path.exists(path):
        meshgen.write_cavity(path, meshgen.CavitySpec(n, re=RE, dt=DT, steps=T_STEPS, ngp=8))
    return path


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(info, klass, iters_per_launch, mixed):
    """Algorithmic HBM bytes of one launch: every matrix entry (value + int32
    column) and every vector read or written once per pass."""
    sv = 4 if mixed else 8
    nnzZ, NNp = info.nnzZ, info.NNp
    if klass in ("pcg64", "pcg32"):
        s = 8 if klass == "pcg64" else 4
        b_z = nnzZ * (s + 4) + 4 * (NNp + 1) + 2 * NNp * s
        b_it = b_z + 9 * NNp * s
        return iters_per_launch * b_it + 6 * NNp * s
    if klass == "step1":
        return (info.nnzK * (sv + 4) + 4 * (info.NN + 1) + info.nnzG * (3 * sv + 4) + 4 * (info.NN + 1)
                + 7 * 3 * info.NN * 8 + NNp * 8)
    if klass == "spmv_k3":
        return info.nnzK * (sv + 4) + 4 * (info.NN + 1) + 2 * 3 * info.NN * 8
    if klass == "gt":
        return info.nnzG * (3 * sv + 4) + 4 * (NNp + 1) + 3 * info.NN * 8 + NNp * 8
    if klass == "step3":
        return info.nnzG * (3 * sv + 4) + 4 * (info.NN + 1) + 7 * 3 * info.NN * 8 + NNp * 8
    if klass == "resid64":
        return nnzZ * 12 + 4 * (NNp + 1) + 4 * NNp * 8
    if klass == "convect":
        return 3 * 3 * info.NN * 8 + info.NE * (27 * 4 + 8 * 3 * 8)
    if klass == "fcg2l":
        # persistent two-level iteration, per iteration: the 125-tap
        # structured Z (the HBM stream) and every vector pass once -- r in
        # the restriction; dinv, r read and z written in the preconditioned
        # residual; z, r, p, q read and w written with the dots; z, w, p, q,
        # x, r read and p, q, x, r written in the update (one stored
        # direction).  The FP16 coarse inverse is not counted: it stays in
        # L2 (coarse_inverse_bytes below).
        return iters_per_launch * (stencil_coef_bytes(info) + 19 * info.NNp * 4)
    if klass == "spmv_z":
        # flexible-CG SpMV w = Z z: the CSR form of Z (values and int32
        # columns, the per-unit bytes of the SpMV) plus z gathered once, w
        # written and r, p, q read for the fused dot products.  In the FP32
        # inner solves the kernel streams Z in its 125-tap structured form
        # instead (format_bytes below): fewer bytes than this count.
        s = 4 if mixed else 8
        return nnzZ * (s + 4) + 4 * (NNp + 1) + 5 * NNp * s
    return 0


def stencil_coef_bytes(info):
    """The 125 FP32 coefficients per row of the structured form of Z, stored
    per 32-row slice."""
    return 125 * 32 * ((info.NNp + 31) // 32) * 4


def coarse_inverse_bytes(nc):
    """The FP16 dense inverse of the coarse matrix, rows padded to 8."""
    return nc * ((nc + 7) // 8 * 8) * 2


def stencil_spmv_bytes(info):
    """Bytes of one flexible-CG SpMV over the 125-tap structured form of Z
    (FP32 coefficients stored per 32-row slice, no column indices) with z
    gathered once, w written and r, p, q read for the fused dot products."""
    return 125 * 32 * ((info.NNp + 31) // 32) * 4 + 5 * info.NNp * 4


# dram__bytes_read.sum + dram__bytes_write.sum of one launch from an ncu
# capture, keyed by (kernel class, pressure nodes, mixed precision), with the
# profile summary it comes from.  Not measured in the bench run itself.
NCU_TRAFFIC = {
    ("spmv_z", 65 ** 3, True): (139.889152e6 + 4.155648e6,
                                "profiles/fcg_twolevel_cavity64.md: ncu --set full, k_fcg_spmv_stencil, "
                                "64^3 cavity, one launch"),
}


def cg_iteration_bytes(info, mixed, structured=False):
    """Algorithmic bytes of one CG iteration: one pass over Z with its
    vectors (the CSR form, values and int32 columns; the 125-tap structured
    form in the FP32 inner solves on a structured grid), plus p, r, x, Ap and
    the diagonal."""
    s = 4 if mixed else 8
    if mixed and structured:
        return 125 * 32 * ((info.NNp + 31) // 32) * 4 + 2 * info.NNp * s + 9 * info.NNp * s
    return info.nnzZ * (s + 4) + 4 * (info.NNp + 1) + 2 * info.NNp * s + 9 * info.NNp * s


def step_bytes(info, steps, subiters, cg_iters, mixed, structured=False):
    """Algorithmic HBM bytes of one time step, averaged over a run: per
    sub-iteration the convection, step1 (K u, G p, update), G^T, step3 and
    about 12 element-wise passes over the FP64 state; per CG iteration
    cg_iteration_bytes; one K Acc pass per sub-iteration that did not end
    its step (subiters - steps, exact when no step ran out)."""
    per_sub = (algorithmic_bytes(info, "convect", 0, mixed) + algorithmic_bytes(info, "step1", 0, mixed)
               + algorithmic_bytes(info, "gt", 0, mixed) + algorithmic_bytes(info, "step3", 0, mixed)
               + 12 * 3 * info.NN * 8)
    kacc = max(0, subiters - steps)
    total = (subiters * per_sub + cg_iters * cg_iteration_bytes(info, mixed, structured)
             + kacc * algorithmic_bytes(info, "spmv_k3", 0, mixed))
    return total / max(1, steps)


def unet_flops(dims):
    """FLOPs of one U-Net application on a pressure grid (multiply-adds of the
    11 convolutions, counted as 2 flops each)."""
    d0 = list(dims)
    lv = [d0, [(v - 1) // 2 + 1 for v in d0]]
    lv.append([(v - 1) // 2 + 1 for v in lv[1]])
    vox = [a[0] * a[1] * a[2] for a in lv]
    convs = [(0, 1, 16), (1, 16, 32), (1, 32, 32), (2, 32, 64), (2, 64, 64), (2, 64, 64), (2, 64, 32),
             (1, 32, 32), (1, 32, 16), (0, 16, 16), (0, 16, 1)]
    return sum(2 * 27 * ci * co * vox[l] for (l, ci, co) in convs)


def rank_barrier(dist) -> None:
    """Barrier over the replicas; nothing to do for one process."""
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x: float, device: str = "cuda") -> float:
    """The largest x over the replicas (every rank times its own GPU; the
    job is as fast as its slowest rank).  device: where the all-reduce
    buffer lives, "cuda" for NCCL, "cpu" for gloo."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, units_per_rank: float, ms_max: float) -> float:
    """Whole-job rate of independent replicas (weak scaling): the units all
    ranks processed over the slowest rank's time in milliseconds."""
    return world * units_per_rank / (ms_max / 1000.0)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import cfdfs

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    work = tempfile.mkdtemp(prefix=f"cfdbench{rank}_")
    deck = make_deck(os.path.join(work, "cavity64.inp"), args.n)
    learned = args.precond == "learned"
    pc_of = {"learned": cfdfs.PC_LEARNED, "twolevel": cfdfs.PC_TWOLEVEL, "jacobi": cfdfs.PC_JACOBI}

    def barrier():
        rank_barrier(dist)

    def ranks_max(x: float) -> float:
        return max_over_ranks(dist, x)

    def timed_solver(precision, precond, steps, warmup, warm=None):
        # --cg-warm 1 (the default) starts the measured path's pressure solves
        # from the previous sub-iteration's pressure increment; the FP64
        # Jacobi-PCG comparison path starts them from x0 = 0, as the reference
        # does (warm=0)
        warm = args.cg_warm if warm is None else warm
        s = cfdfs.Solver(device=local_rank, precision=precision, cg_rtol=1e-8, cg_maxit=args.cg_maxit,
                         precond=pc_of[precond], fcg_net_iters=args.net_iters, cg_warm=warm,
                         inner_rtol=args.inner_rtol)
        t0 = time.time()
        s.load(deck)
        t1 = time.time()
        s.step0()
        t2 = time.time()
        if precond == "learned":
            s.load_unet(args.weights)
        if precond != "jacobi":
            s.precond_apply(np.zeros(s.refresh().NNp))  # builds the coarse space (set-up)
        t3 = time.time()
        setup_s = t3 - t0
        # deck reading and host preprocessing (numbering, patterns) plus the
        # upload; step0's operator assembly on the device; the network's
        # weights and the coarse space (Galerkin product, factorisation)
        setup_parts = {"load": round(t1 - t0, 3), "step0": round(t2 - t1, 3), "precond": round(t3 - t2, 3)}
        for _ in range(warmup):
            s.run(1)
        if steps == 0:
            return s, dict(setup_s=setup_s, setup_parts=setup_parts)
        stream = torch.cuda.ExternalStream(s.stream_ptr, device=local_rank)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = s.launch_count()
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local_rank) as clk:
            ev0.record(stream)
            st = s.run(steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        launches = s.launch_count() - n0
        return s, dict(ms=ms, st=st, launches=launches, clocks=clk.summary(), setup_s=setup_s,
                       setup_parts=setup_parts)

    precision = cfdfs.MIXED if args.precision == "mixed" else cfdfs.FP64
    # the cavity's pressure nodes form an identity-numbered cube, so the
    # coarse-space preconditioners run their FP32 inner solves on the
    # structured form of Z
    structured = args.precond in ("twolevel", "learned")
    s, r = timed_solver(precision, args.precond, args.steps, args.warmup)
    info = s.refresh()
    ms_max = ranks_max(r["ms"])
    value = replica_rate(world, args.steps, ms_max)

    # the same precision with the two-level preconditioner alone (the learned
    # preconditioner without its network): what the network adds
    twolevel = None
    if learned and args.fp64_steps:
        s2, r2 = timed_solver(precision, "twolevel", args.steps, args.warmup)
        ms2 = ranks_max(r2["ms"])
        twolevel = dict(steps_per_s=round(replica_rate(world, args.steps, ms2), 4), ms_per_step=round(ms2 / args.steps, 3),
                        cg_iters_per_step=round(r2["st"].cg_iters / max(1, r2["st"].steps), 1))
        s2.close()

    # the plain FP64 Jacobi-PCG path on the same workload and the same steps
    # (denominator of the headline target, and the accuracy reference)
    fp64, acc = None, None
    if args.fp64_steps and not (precision == cfdfs.FP64 and args.precond == "jacobi"):
        s64, r64 = timed_solver(cfdfs.FP64, "jacobi", args.steps, args.warmup, warm=0)
        ms64 = ranks_max(r64["ms"])
        fp64 = dict(steps=args.steps, steps_per_s=round(replica_rate(world, args.steps, ms64), 4),
                    ms_per_step=round(ms64 / args.steps, 3), cg_x0="zero",
                    cg_iters_per_step=round(r64["st"].cg_iters / max(1, r64["st"].steps), 1))
        U1, P1 = s.state()
        U0, P0 = s64.state()
        d1, d0 = s.vector("DIV"), s64.vector("DIV")
        rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        acc = {"u_rel_l2": rel(U1, U0), "p_rel_l2": rel(P1, P0), "div_max": float(np.abs(d1).max()),
               "div_max_fp64": float(np.abs(d0).max()),
               "vs": f"FP64 Jacobi-PCG GPU path after the same {args.warmup + args.steps} steps (that path "
                     f"matches the FP64 oracle to <= 1e-6 per field in the parity tests)"}
        s64.close()

    # e2e through the C ABI with host buffers, on the same steps as the timed
    # region above: a fresh solver with the same options runs the same W
    # warm-up steps from rest, then for each of the K timed steps the state
    # goes host -> device from pinned memory (cfd_upload_state), one step
    # runs (cfd_run(1)) and the new state comes back (cfd_download_state).
    # Events around cfd_run alone give the device time of those same steps.
    s_e, _ = timed_solver(precision, args.precond, 0, args.warmup)
    U = torch.empty(3 * info.NN, dtype=torch.float64, pin_memory=True).numpy()
    P = torch.empty(info.NNp, dtype=torch.float64, pin_memory=True).numpy()
    s_e.state(out=(U, P))
    stream_e = torch.cuda.ExternalStream(s_e.stream_ptr, device=local_rank)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream_e)
    for k in range(args.steps):
        s_e.set_state(U, P)
        evs[k][0].record(stream_e)
        s_e.run(1)
        evs[k][1].record(stream_e)
        s_e.state(out=(U, P))
    ev1.record(stream_e)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = ranks_max(ev0.elapsed_time(ev1))
    e2e_value = replica_rate(world, args.steps, e2e_ms)
    e2e_dev_ms = ranks_max(sum(a.elapsed_time(b) for a, b in evs))
    s_e.close()
    state_bytes = (3 * info.NN + info.NNp) * 8

    # per-kernel-class event timing on a separate short pass (events around
    # every launch would perturb the timed region), and the roofline of the
    # dominant class
    s.profile(True)
    s.run(args.profile_steps)
    prof = s.profile_read()
    s.profile(False)
    # roofline of the dominant kernel class with a stated byte (or flop) count
    phases = s.profile_fcg2l()
    known = ("pcg32", "pcg64", "spmv_z", "fcg2l", "unet", "step1", "spmv_k3", "gt", "step3", "resid64", "convect")
    top = max((k for k in prof if k in known), key=lambda k: prof[k]["ms"])
    p = prof[top]
    its_per_launch = (p["iters"] / p["launches"]) if p["launches"] else 0
    avg_ms = p["ms"] / max(1, p["launches"])
    peak, peak_kind = peaks()
    if top == "unet":
        m = round(info.NNp ** (1 / 3))
        alg = unet_flops((m, m, m))
        tpeak, tkind = tensor_peak()
        achieved = alg / (avg_ms / 1000.0) / 1e12 if avg_ms > 0 else 0.0
        roof = {"bound": "tensor", "kernel": top, "achieved": round(achieved, 2), "peak": tpeak, "unit": "TFLOP/s",
                "frac": round(achieved / tpeak, 4), "peak_kind": f"{tkind} bf16_tflops",
                "algorithmic_flops_per_launch": int(alg), "avg_launch_ms": round(avg_ms, 4), "traffic": None}
    else:
        mixed = precision == cfdfs.MIXED
        alg = algorithmic_bytes(info, top, its_per_launch, mixed)
        csr = None
        if top == "spmv_z" and mixed and structured:
            # the FP32 inner solves stream Z in its 125-tap structured form
            # (no column indices): those are the bytes the kernel moves and
            # the fraction is taken on them; the CSR count of the same
            # product stays beside it under its own name
            csr = alg
            alg = stencil_spmv_bytes(info)
        achieved = alg / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else 0.0
        roof = {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs",
                "algorithmic_bytes_per_launch": int(alg), "avg_launch_ms": round(avg_ms, 4),
                "iters_per_launch": round(its_per_launch, 1), "traffic": None}
        if csr is not None:
            roof["bytes_basis"] = "125-tap structured Z (FP32 values, no column indices) + 5 vector passes"
            roof["csr_equivalent_bytes_per_launch"] = int(csr)
            roof["csr_equivalent_achieved"] = round(csr / (avg_ms / 1000.0) / 1e9, 1) if avg_ms > 0 else 0.0
        if top == "fcg2l":
            roof["bytes_basis"] = ("per iteration: 125-tap structured Z + 19 FP32 vector passes; the FP16 coarse "
                                   "inverse (L2-resident) is not counted")
            iters = max(1, p["iters"])
            ph = {k: round(v / iters * 1000.0, 2) for k, v in phases.items()}  # us per iteration
            roof["phases_us_per_iter"] = ph
            spmv_b = stencil_spmv_bytes(info)
            if ph.get("spmv", 0) > 0:
                # the SpMV phase alone on its own bytes (first block's clock)
                ach = spmv_b / (ph["spmv"] * 1e-6) / 1e9
                roof["spmv_phase"] = {"bytes": int(spmv_b), "us": ph["spmv"], "achieved": round(ach, 1),
                                      "frac": round(ach / peak, 4)}
        t = NCU_TRAFFIC.get((top, info.NNp, mixed))
        if t is not None:
            roof["traffic"] = int(t[0])
            roof["traffic_source"] = t[1]
    # the whole step on the same algorithmic byte counts, with the timed
    # run's own sub-iteration and CG iteration counts
    st_t = r["st"]
    b_step = step_bytes(info, st_t.steps, st_t.subiters, st_t.cg_iters, precision == cfdfs.MIXED, structured)
    step_ach = b_step / (ms_max / args.steps / 1000.0) / 1e9
    step_roof = {"bound": "hbm", "bytes_per_step": int(b_step), "achieved": round(step_ach, 1), "peak": peak,
                 "unit": "GB/s", "frac": round(step_ach / peak, 6), "peak_kind": f"{peak_kind} hbm_gbs"}
    total_ms = sum(v["ms"] for v in prof.values())
    kernels = {k: dict(launches=v["launches"], ms=round(v["ms"], 3),
                       share=round(v["ms"] / total_ms, 4) if total_ms else 0.0,
                       iters=v["iters"]) for k, v in prof.items() if v["launches"]}
    s.close()

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and args.cpu_baseline:
            cpu = cpu_baseline(deck, args.n, budget_s=args.cpu_budget)
        out = {
            "metric": METRIC,
            "value": round(value, 4),
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("f32+f64" if precision == cfdfs.MIXED else "f64") + ("+bf16" if learned else ""),
            "data": "synthetic: generated structured cavity deck (no dataset); fluid starts at rest",
            "config": {"workload": workload(args.n), "elements": args.n ** 3, "precision": args.precision,
                       "precond": {"learned": "Jacobi + coarse space + learned U-Net correction in flexible CG "
                                   f"(network in the first {args.net_iters or 'every'} iteration(s) of each solve; "
                                   "Jacobi-PCG fallback)",
                        "twolevel": "Jacobi + Galerkin coarse-space correction (17^3 lattice) in CG",
                        "jacobi": "jacobi"}[args.precond],
                       "weights": os.path.relpath(args.weights, ROOT) if learned else None,
                       "ngp": 8, "cg_rtol": 1e-8, "cg_x0": "previous increment" if args.cg_warm else "zero",
                       "inner_rtol": args.inner_rtol if precision == cfdfs.MIXED else None,
                       "timed_steps": f"steps {args.warmup + 1}..{args.warmup + args.steps} of the run from rest",
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (no flush needed)",
                       "setup_s": round(r["setup_s"], 2), "setup_parts_s": r["setup_parts"]},
            "cg_iters_per_step": round(r["st"].cg_iters / max(1, r["st"].steps), 1),
            "subiters_per_step": round(r["st"].subiters / max(1, r["st"].steps), 2),
            "pressure_fallbacks": int(r["st"].fallbacks),  # solves that fell back to Jacobi-PCG
            "fp64_path": fp64,
            "twolevel_path": twolevel,
            "speedup_vs_fp64": round(value / fp64["steps_per_s"], 3) if fp64 else None,
            "accuracy": acc,
            "roofline": roof,
            "step_roofline": step_roof,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 4), "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": args.steps,
                    "timed_steps": f"steps {args.warmup + 1}..{args.warmup + args.steps} of a fresh run from rest "
                                   f"(the same steps as value)",
                    "device_steps_per_s_same_steps": round(replica_rate(world, args.steps, e2e_dev_ms), 4),
                    "path": "C ABI: cfd_upload_state + cfd_run(1) + cfd_download_state, pinned host buffers"},
            "gpu_launches": r["launches"],
            "clocks": r["clocks"],
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


REF_EXE = os.path.join(ROOT, "oracle", "_ref", "fs_ref")
REF_THREADS = 8  # N_OPENMP_THREADS and N_MKL_THREADS, blascoCodinaHuerta.cpp:85-86


def ref_cores() -> int:
    return min(REF_THREADS, os.cpu_count() or 1)


def run_reference_binary(n, warm, timed, budget_s=None, timeout_s=1200):
    """Runs the reference's own program on the n^3 cavity deck for up to
    warm + timed time steps (its while (timeT < t_final) loop, t_final set
    in the deck) and returns the wall times it prints itself for the timed
    steps in the TimeSpend column of its monitor table
    (blascoCodinaHuerta.cpp:2855-3093, gettimeofday around each step), plus
    the wall time of the process (set-up included).  The program runs in a
    pseudo-terminal so that its monitor rows arrive as it prints them; with
    a budget it is stopped once the timed steps it finished exceed that many
    seconds (at least one timed step)."""
    import pty
    import select
    from cfdfs import meshgen
    work = tempfile.mkdtemp(prefix="cfdbench_fsref_")
    meshgen.write_cavity(os.path.join(work, "cavity.inp"),
                         meshgen.CavitySpec(n, re=RE, dt=DT, steps=warm + timed, ngp=8))
    with open(os.path.join(work, "ProblemName.txt"), "w") as f:
        f.write("cavity\n")
    rows, buf = [], b""
    t0 = time.time()
    master, slave = pty.openpty()
    proc = subprocess.Popen([REF_EXE], cwd=work, stdin=subprocess.DEVNULL, stdout=slave, stderr=slave)
    os.close(slave)
    stopped = False
    try:
        while True:
            if time.time() - t0 > timeout_s:
                raise RuntimeError("reference program exceeded its time limit")
            ready, _, _ = select.select([master], [], [], 1.0)
            if not ready:
                if proc.poll() is not None:
                    break
                continue
            try:
                chunk = os.read(master, 65536)
            except OSError:
                break
            if not chunk:
                break
            buf += chunk
            *lines, buf = buf.split(b"\n")
            for line in lines:
                parts = line.decode(errors="replace").split()
                if len(parts) == 9 and parts[0].isdigit() and parts[1].isdigit():
                    rows.append([float(x) for x in parts])
            done = rows[warm:]
            if budget_s is not None and done and sum(r[7] for r in done) > budget_s and len(rows) < warm + timed:
                proc.kill()
                stopped = True
                break
    finally:
        os.close(master)
        proc.wait()
    wall = time.time() - t0
    if not stopped and proc.returncode != 0:
        raise RuntimeError(f"reference program failed ({proc.returncode})")
    times = [r[7] for r in rows[warm:warm + timed]]
    if not times:
        raise RuntimeError("reference program printed no timed monitor row")
    return times, wall


def cpu_baseline(deck, n, budget_s=40.0, threads=0):
    """The reference's own CPU solver (oracle/_ref/fs_ref) on a bounded
    sample of the same workload: one warm-up time step from rest, then two
    timed steps (steps 2..3 of the run; the reference arm times steps
    2..K+1 of the same run).  Where that binary was not built, the oracle
    (the C++ FP64 restatement, all host threads) runs instead."""
    if os.path.exists(REF_EXE):
        times, wall = run_reference_binary(n, 1, 2)
        return {"value": round(len(times) / sum(times), 5), "unit": "steps/s", "cores": ref_cores(),
                "kind": "reference",
                "sample": f"time steps 2..3 from rest of the same {n}^3 deck, timed by the reference program "
                          f"itself (its TimeSpend column); the unmodified blascoCodinaHuerta.cpp with "
                          f"self-written MKL/CSparse stand-ins, the {REF_THREADS} OpenMP/MKL threads it sets; "
                          f"set-up excluded (whole process {wall:.1f} s)",
                "seconds": round(sum(times), 2)}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build()
    o = pyoracle.Oracle(deck, threads=threads)
    t0 = time.time()
    o.step0()
    setup = time.time() - t0
    o.run(1)
    steps, t0 = 0, time.time()
    while steps < 2 or (time.time() - t0 < budget_s * 0.5 and steps < 2):
        o.run(1)
        steps += 1
    el = time.time() - t0
    o.close()
    return {"value": round(steps / el, 5), "unit": "steps/s", "cores": pyoracle.threads(), "kind": "port",
            "sample": f"time steps 2..{steps + 1} from rest of the same {n}^3 deck, FP64 Jacobi-PCG rtol 1e-8 "
                      f"(the reference program was not built); set-up ({setup:.1f} s) excluded",
            "seconds": round(el, 2)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    n = args.n
    base = {"impl": "reference", "metric": METRIC, "unit": "steps/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: generated structured cavity deck; fluid starts at rest",
            "config": {"workload": workload(n), "precision": "fp64", "ngp": 8,
                       "cg": "MKL dcg Jacobi-PCG, x0 = 0, |r|^2 <= 1e-12 |b|^2 (the reference's own settings)"}}
    if os.path.exists(REF_EXE):
        warm = 1
        times, wall = run_reference_binary(n, warm, args.steps, budget_s=args.cpu_budget)
        v = len(times) / sum(times)
        cores = ref_cores()
        cpu = {"value": round(v, 5), "unit": "steps/s", "cores": cores, "kind": "reference",
               "sample": f"time steps {warm + 1}..{warm + len(times)} from rest of the {n}^3 deck (timed steps capped at "
                         f"{args.cpu_budget:.0f} s), each timed by the "
                         f"reference program itself (TimeSpend column): the unmodified "
                         f"fractionalStep/Cpp/blascoCodinaHuerta.cpp built with self-written MKL/CSparse "
                         f"stand-ins, {REF_THREADS} OpenMP and MKL threads as it sets them; whole process "
                         f"{wall:.1f} s including its set-up"}
        out = dict(base, value=round(v, 5), steps=len(times), warmup=warm, ms_per_step=round(1000 / v, 1),
                   cpu_baseline=cpu)
    else:
        work = tempfile.mkdtemp(prefix="cfdbench_ref_")
        deck = make_deck(os.path.join(work, "cavity64.inp"), n)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        pyoracle.build()
        o = pyoracle.Oracle(deck)
        o.step0()
        o.run(1)
        steps, t0 = 0, time.time()
        while steps < args.steps and (steps < 1 or time.time() - t0 < args.cpu_budget):
            o.run(1)
            steps += 1
        el = time.time() - t0
        o.close()
        v = steps / el
        cpu = {"value": round(v, 5), "unit": "steps/s", "cores": pyoracle.threads(), "kind": "port",
               "sample": f"time steps 2..{steps + 1} of the {n}^3 deck on the oracle (the reference program was not "
                         f"built on this machine)"}
        out = dict(base, value=round(v, 5), steps=steps, warmup=1, ms_per_step=round(1000 * el / steps, 1),
                   cpu_baseline=cpu)
    out["e2e"] = {"value": out["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--n", type=int, default=N_ELEM, help="elements per side (64 = the headline workload)")
    ap.add_argument("--precond", default=None, choices=["learned", "twolevel", "jacobi"],
                    help="default: learned when the weight file exists, else twolevel")
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--net-iters", type=int, default=1,
                    help="learned preconditioner: network in the first this-many iterations of a solve (0 = all)")
    ap.add_argument("--fp64-steps", type=int, default=1, help="0 skips the FP64 Jacobi-PCG comparison run")
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--cg-maxit", type=int, default=5000)
    ap.add_argument("--inner-rtol", type=float, default=1e-5,
                    help="mixed precision: relative tolerance of each FP32 inner solve of the FP64 refinement")
    ap.add_argument("--cg-warm", type=int, default=1,
                    help="1: the measured path's pressure solves start from the previous sub-iteration's "
                         "increment; 0: from x0 = 0 (the reference's choice, always used by the FP64 comparison)")
    ap.add_argument("--cpu-budget", type=float, default=90.0,
                    help="seconds of timed reference steps before the reference arm stops")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.precond is None:
        args.precond = "learned" if os.path.exists(args.weights) else "twolevel"
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    else:
        out = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
