"""Benchmark: Mcell-steps/s of the SSP-RK3 / WENO-5 / MG-PCG step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tgv64] [--precision fp64|mixed]

One step = one full SSP-RK3 step (three RHS evaluations, three projections
solved by MG-PCG to the case tolerance) over the whole case. Prints one JSON
line on rank 0. N > 1 runs one independent replica per GPU (the path does not
shard: no collective on the data path); the time is the max over ranks.

`value` is device-timed with CUDA events on the case's stream with the state
resident in HBM; the L2 is flushed (a 256 MiB write) between timed steps.
`e2e` is the same metric through the C ABI with host buffers: the state is
uploaded from pinned memory, stepped and downloaded every step.
`--impl reference` times the reference's own CPU implementation (oracle/_ref,
compiled from the reference sources) on this host's cores on the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "nabla-ai_b200"))

METRIC = "Mcell-steps/s (mixed vs FP64 plain, div<1e-8) on 1 B200; p50/p99 solve latency"
UNIT = "Mcell-steps/s"
FAMILIES = ["rhs_rk", "smooth", "resid_restrict", "coarse_cg", "pcg_matvec", "pcg_update",
            "pcg_center", "pcg_mean", "pcg_dots", "pcg_dir", "div", "correct", "diag"]


def workload(name):
    from nabla_b200 import cases
    if name == "tgv64":
        g, cfg = cases.taylor_green(64)
        st = cases.taylor_green_state(g)
        desc = ("Taylor-Green vortex, periodic [0,2pi]^3, uniform 64^3 MAC grid (512 bricks of 8^3), "
                "nu=1/1600, WENO-5, fixed dt=computeDt at CFL 0.4, MG-PCG to 1e-10")
        return g, cfg, st, desc
    raise SystemExit(f"unknown workload {name}")


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(REPO, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import numpy as np
    import torch

    from nabla_b200 import abi, solver

    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    g, cfg, st, desc = workload(args.workload)
    ns = solver.NSSolver(g, cfg, precision=prec, ctx=ctx)
    ns.set_state(*st)
    dt = ns.compute_dt()
    cells = ns.cell_count
    stream = torch.cuda.ExternalStream(ns.ctx.lib.nb_case_stream(ns.h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")

    def one_step():
        return ns.step(dt)

    # warm-up
    for _ in range(args.warmup):
        rep = one_step()
    torch.cuda.synchronize()
    # share of each kernel family (one profiled step per family, untimed)
    shares = {}
    for fam in (FAMILIES if args.shares else ["smooth"]):
        ctx.lib.nb_ctx_profile(ctx.h, fam.encode())
        one_step()
        ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
        ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
        shares[fam] = {"ms": ms.value, "launches": nl.value, "bytes": nb.value}
    ctx.lib.nb_ctx_profile(ctx.h, None)
    total = sum(v["ms"] for v in shares.values()) or 1.0
    top = max(shares, key=lambda k: shares[k]["ms"])
    # timed region: K steps, each bracketed by events on the case stream,
    # L2 flushed between steps outside the events; the top family profiled
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    elapsed = 0.0
    reps = []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            reps.append(one_step())
            e1.record(stream)
            e1.synchronize()
            elapsed += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    # Roofline of the dominant kernel family: the same K steps again, issued
    # as direct launches with CUDA events around every launch of that family
    # (events cannot sit inside the graph's device-side MG-PCG loop).
    ctx.lib.nb_ctx_profile(ctx.h, top.encode())
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        one_step()
    torch.cuda.synchronize()
    ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
    ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
    ctx.lib.nb_ctx_profile(ctx.h, None)
    t = torch.tensor([elapsed], dtype=torch.float64, device=f"cuda:{local_rank}")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    elapsed_max = float(t.item())
    value = world * cells * args.steps / (elapsed_max * 1e-3) / 1e6
    # end to end through the C ABI with host buffers (pinned)
    pinned = [torch.from_numpy(a.copy()).pin_memory().numpy() for a in ns.get_state()]
    outs = [torch.empty(a.size, dtype=torch.float64).pin_memory().numpy() for a in pinned]
    n_e2e = max(2, args.steps // 2)
    e2e_ms = 0.0
    for _ in range(n_e2e):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ns.set_state(*pinned)
        ns.step(dt)
        st_ = ns.get_state()
        for o, s in zip(outs, st_):
            o[:] = s
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local_rank}")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_value = world * cells * n_e2e / (float(te.item()) * 1e-3) / 1e6
    hbm, peak_kind = peaks()
    achieved = (nb.value / (ms.value * 1e-3) / 1e9) if ms.value > 0 else 0.0
    per_launch_bytes = nb.value / max(nl.value, 1)
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == abi.PRECISION_FP64 else "f32+f64",
        "data": "synthetic (analytic Taylor-Green initial state)",
        "config": {"workload": desc, "cells": cells, "precision": args.precision,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed between timed steps (256 MiB write); working set < L2",
                   "poisson_cycles_per_step": reps[-1].poisson_iters},
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(sum(a.nbytes for a in pinned)),
                "d2h_bytes_per_step": int(sum(a.nbytes for a in outs))},
        "gpu_launches": int(launches),
        "roofline": {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 5),
                     "bytes_per_launch": per_launch_bytes, "launches": int(nl.value),
                     "avg_launch_us": round(ms.value * 1e3 / max(nl.value, 1), 3), "traffic": None},
        "kernel_shares": {k: round(v["ms"] / total, 4) for k, v in sorted(shares.items(),
                                                                         key=lambda kv: -kv[1]["ms"])},
        "divergence_max": reps[-1].divergence_max,
        "clocks": clk.summary(),
    }
    return out


def cpu_sample(args, steps):
    """The reference's CPU step on this host (oracle/_ref); returns s/step."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    g, cfg, st, _ = workload(args.workload)
    ref = oracle.Reference()
    ns = ref.ns(g, cfg)
    ns.set_state(*st)
    dt = ns.compute_dt()
    t0 = time.perf_counter()
    for _ in range(steps):
        ns.step(dt)
    return (time.perf_counter() - t0) / steps, g.ncell


def _ref_worker(q, args_dict, steps, warmup):
    a = argparse.Namespace(**args_dict)
    if warmup:
        cpu_sample(a, warmup)
    s, cells = cpu_sample(a, steps)
    q.put((s, cells))


def run_reference(args):
    """Reference arm: the reference's serial CPU step run as one independent
    case per host core (it has no threading), aggregate Mcell-steps/s."""
    import multiprocessing as mp
    cores = int(os.environ.get("NB_REF_CORES", min(os.cpu_count() or 1, 16)))
    steps = max(1, args.steps)
    ctxm = mp.get_context("spawn")
    q = ctxm.Queue()
    procs = [ctxm.Process(target=_ref_worker, args=(q, vars(args), steps, min(args.warmup, 1)))
             for _ in range(cores)]
    t0 = time.perf_counter()
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    wall = time.perf_counter() - t0
    s_per_step = max(r[0] for r in res)
    cells = res[0][1]
    value = cores * cells / s_per_step / 1e6
    _, _, _, desc = workload(args.workload)
    return {
        "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(s_per_step * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic Taylor-Green initial state)", "impl": "reference",
        "config": {"workload": desc, "cells": cells, "precision": "fp64"},
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{steps} NSSolver::step per process, {cores} independent processes"},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv64")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--shares", type=int, default=1,
                    help="1: time each kernel family once before the timed region")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0:
        if args.cpu_steps > 0:
            s, cells = cpu_sample(args, args.cpu_steps)
            out["cpu_baseline"] = {"value": round(cells / s / 1e6, 5), "unit": UNIT, "cores": 1,
                                   "kind": "reference",
                                   "sample": f"{args.cpu_steps} NSSolver::step of the same case, 1 thread"}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
