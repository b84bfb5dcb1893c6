"""Benchmark: Mcell-steps/s of the SSP-RK3 / WENO-5 / MG-PCG step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload channel3|tgv64] [--precision fp64|mixed]

Workloads (seeded synthetic inputs, no datasets):
  channel3  3-level octree obstacle channel, [0,4]x[0,1]^2, base 64x16x16 in 8^3
            bricks refined to effective 256x64x64 where the initial vorticity is in
            its top fifth or near the 6 seeded boxes; inflow U=1, outlet, walls,
            nu=1/1000, CFL 0.4 (dt from the CFL condition every step). Default.
  tgv64     Taylor-Green vortex on the periodic 64^3 box, nu=1/1600, fixed dt.

One step = one full SSP-RK3 step (three RHS evaluations, three projections
solved by MG-PCG to 1e-10) over every leaf cell. Prints one JSON line on rank
0. N > 1 runs one independent replica per GPU (the path does not shard: no
collective on the data path); the time is the max over ranks.

`value` is device-timed with CUDA events on the case's stream with the state
resident in HBM; the L2 is flushed (a 256 MiB write) between timed steps. For
the octree workload both arithmetic forms are timed (`forms`); `value` is the
form named by --precision (mixed by default there) and `accuracy` states the
mixed form's velocity / pressure / divergence error against the FP64 form.
`e2e` is the same metric through the C ABI with host buffers: the state is
uploaded from pinned memory, stepped and downloaded every step.
`--impl reference` times the reference's own CPU implementation (oracle/_ref,
compiled from the reference sources) on this host's cores; the reference has no
octree MAC step, so for channel3 it runs its uniform NSSolver on the
uniform-fine (256x64x64) version of the same case.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "nabla-ai_b200"))

METRIC = "Mcell-steps/s (mixed vs FP64 plain, div<1e-8) on 1 B200; p50/p99 solve latency"
UNIT = "Mcell-steps/s"
# DRAM bytes (read + write) per launch of a kernel family, averaged over the
# same launches the roofline averages, from one ncu capture of this workload
# (profiles/channel3_launches_and_captures.md: 40 consecutive k_smooth launches).
NCU_TRAFFIC = {("channel3", "smooth"): 2.159e6}
FAMILIES = ["rhs_rk", "vgrid", "smooth", "resid_restrict", "coarse_cg", "vtail", "pcg_matvec", "pcg_update",
            "pcg_center", "pcg_mean", "pcg_dots", "div", "correct", "diag", "sync"]


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
class UniformRun:
    """A uniform-grid case through nb_case_* (fixed dt from the initial state)."""

    def __init__(self, ctx, prec):
        from nabla_b200 import cases, solver
        g, cfg = cases.taylor_green(64)
        self.ns = solver.NSSolver(g, cfg, precision=prec, ctx=ctx)
        self.ns.set_state(*cases.taylor_green_state(g))
        self.dt = self.ns.compute_dt()
        self.cells = self.ns.cell_count
        self.h = self.ns.h
        self.desc = ("Taylor-Green vortex, periodic [0,2pi]^3, uniform 64^3 MAC grid (512 bricks of 8^3), "
                     "nu=1/1600, WENO-5, fixed dt=computeDt at CFL 0.4, MG-PCG to 1e-10")
        self.data = "synthetic (analytic Taylor-Green initial state)"

    def step(self):
        return self.ns.step(self.dt)

    def get_state(self, out=None):
        return self.ns.get_state(out)

    def set_state(self, *st):
        self.ns.set_state(*st)


_CHANNEL = {}


def channel_workload(seed=0):
    from nabla_b200 import workloads
    if seed not in _CHANNEL:
        _CHANNEL[seed] = workloads.obstacle_channel(seed)
    return _CHANNEL[seed]


class AmrRun:
    """The octree obstacle channel through nb_amr_case_* (CFL dt every step)."""

    def __init__(self, ctx, prec, mesh=None):
        from nabla_b200 import amr
        w = channel_workload()
        self.mesh = mesh or amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
        self.case = amr.AmrCase(self.mesh, w.config, precision=prec)
        self.case.set_state(*w.initial_state(self.case))
        self.cells = self.case.cell_count
        self.h = self.case.h
        self.desc = w.description
        self.data = "synthetic (seeded boxes and random-potential perturbation, seed 0)"

    def step(self):
        return self.case.step(0.0)

    def get_state(self, out=None):
        return self.case.get_state(out)

    def set_state(self, *st):
        self.case.set_state(*st)


def make_run(name, ctx, prec, mesh=None):
    if name == "tgv64":
        return UniformRun(ctx, prec)
    if name == "channel3":
        return AmrRun(ctx, prec, mesh)
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
        fd, self.path = tempfile.mkstemp(prefix="nb_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
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
        self.lines = open(self.path).read().splitlines() if os.path.exists(self.path) else []
        try:
            os.unlink(self.path)
        except OSError:
            pass

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
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


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def timed_steps(run, steps, stream, flush, clock=None):
    """K steps, each bracketed by CUDA events on the case stream; the L2 is
    flushed before every step outside the events. Returns (ms total, reports)."""
    import torch
    elapsed, reps = 0.0, []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps.append(run.step())
        e1.record(stream)
        e1.synchronize()
        elapsed += e0.elapsed_time(e1)
    return elapsed, reps


def profile_step(ctx, run, fam):
    import ctypes as C
    ctx.lib.nb_ctx_profile(ctx.h, fam.encode())
    try:
        run.step()
    finally:
        ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
        ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
        ctx.lib.nb_ctx_profile(ctx.h, None)
    return ms.value, nl.value, nb.value


def max_over_ranks(x, world, device):
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def rel_err(a, b):
    import numpy as np
    den = float(np.abs(b).max()) if b.size else 0.0
    return float(np.abs(a - b).max()) / max(den, 1e-300)


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from nabla_b200 import abi, solver

    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    if args.tuning:
        ctx.set_tuning(**args.tuning)
    precision = args.precision or ("mixed" if args.workload == "channel3" else "fp64")
    prec = abi.PRECISION_MIXED if precision == "mixed" else abi.PRECISION_FP64
    run = make_run(args.workload, ctx, prec)
    cells = run.cells
    stream = torch.cuda.ExternalStream(ctx.lib.nb_case_stream(run.h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    for _ in range(args.warmup):
        run.step()
    torch.cuda.synchronize()
    # share of each kernel family (one profiled direct-launch step per family, untimed)
    shares = {}
    for fam in (FAMILIES if args.shares else ["smooth"]):
        ms, nl, nb = profile_step(ctx, run, fam)
        shares[fam] = {"ms": ms, "launches": nl, "bytes": nb}
    total = sum(v["ms"] for v in shares.values()) or 1.0
    top = max(shares, key=lambda k: shares[k]["ms"])
    # the state the timed steps start from (the end-to-end pass replays the same trajectory)
    start = [torch.from_numpy(a.copy()).pin_memory().numpy() for a in run.get_state()]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    with ClockSampler(local_rank) as clk:
        elapsed, reps = timed_steps(run, args.steps, stream, flush)
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    if world > 1:
        torch.distributed.barrier()
    elapsed_max = max_over_ranks(elapsed, world, device)
    value = world * cells * args.steps / (elapsed_max * 1e-3) / 1e6
    # Roofline of the dominant kernel family: K more steps issued as direct
    # launches with CUDA events around every launch of that family (events
    # cannot sit inside the graph's device-side MG-PCG loop).
    ctx.lib.nb_ctx_profile(ctx.h, top.encode())
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        run.step()
    torch.cuda.synchronize()
    ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
    ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
    ctx.lib.nb_ctx_profile(ctx.h, None)
    # End to end through the C ABI with host buffers (pinned): the same K steps
    # from the same starting state as the timed region, every step uploading
    # the state from host memory and reading the stepped state back into it.
    host = start
    e2e_ms, e2e_cycles = 0.0, 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run.set_state(*host)
        r = run.step()
        run.get_state(host)  # straight back into the pinned buffers
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_cycles += r.poisson_iters
    e2e_value = world * cells * args.steps / (max_over_ranks(e2e_ms, world, device) * 1e-3) / 1e6
    pinned = outs = host
    hbm, peak_kind = peaks()
    achieved = (nb.value / (ms.value * 1e-3) / 1e9) if ms.value > 0 else 0.0
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == abi.PRECISION_FP64 else "f32+f64",
        "data": run.data,
        "config": {"workload": run.desc, "cells": cells, "precision": precision, "tuning": ctx.tuning,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed between timed steps (256 MiB write); working set < L2",
                   "poisson_cycles_per_step": reps[-1].poisson_iters,
                   "poisson_cycles_timed": sum(r.poisson_iters for r in reps)},
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(sum(a.nbytes for a in pinned)),
                "d2h_bytes_per_step": int(sum(a.nbytes for a in outs)),
                "steps": args.steps, "poisson_cycles": e2e_cycles,
                "trajectory": "the timed steps replayed from the same starting state, state uploaded from and "
                              "read back to pinned host memory every step"},
        "gpu_launches": int(launches),
        "roofline": {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 5),
                     "bytes_per_launch": nb.value / max(nl.value, 1), "launches": int(nl.value),
                     "avg_launch_us": round(ms.value * 1e3 / max(nl.value, 1), 3),
                     "traffic": NCU_TRAFFIC.get((args.workload, top))},
        "kernel_shares": {k: round(v["ms"] / total, 4) for k, v in sorted(shares.items(),
                                                                         key=lambda kv: -kv[1]["ms"])},
        "divergence_max": max(r.divergence_max for r in reps),
        "converged": all(bool(r.converged) for r in reps),
        "clocks": clk.summary(),
    }
    if args.workload == "channel3":
        out["forms"], out["accuracy"] = other_form_and_accuracy(args, ctx, run, prec, precision, value,
                                                                stream, flush, world, device)
        if args.same_case_steps > 0:
            out["same_case_as_reference_arm"] = same_case_as_reference(args, ctx, flush, world, device)
        if args.large_steps > 0:
            out["large_case"] = large_case(args, ctx, flush, world, device)
        if args.batch_steps > 0:
            out["batch"] = batch_key(args, rank, world, local_rank)
        if args.serve_seconds > 0:
            srv = serve_once(args, ctx, prec, 7 + rank, args.serve_seconds + args.serve_grace)
            out["serving"] = {"workload": serve_config(args), "precision": precision,
                              **{k: (round(v, 4) if isinstance(v, float) else v) for k, v in srv.items()}}
            out["latency"] = {"p50_s": round(srv["p50_latency_s"], 4), "p99_s": round(srv["p99_latency_s"], 4),
                              "served": srv["served"], "arrived": srv["arrived"],
                              "note": "arrival-to-result latency of the served requests of the `serving` run"}
    return out


def same_case_as_reference(args, ctx, flush, world, device):
    """Both forms on exactly the case the reference arm steps: the uniform-fine
    256x64x64 version of the channel (dt from the CFL condition every step)."""
    import torch

    from nabla_b200 import abi, solver, workloads
    g, cfg, st = workloads.channel_uniform(0)
    out = {"workload": "uniform-fine 256x64x64 obstacle channel (the reference arm's case), "
                       "from its initial state", "cells": g.ncell, "steps": args.same_case_steps}
    for name, prec in (("fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
        ns = solver.NSSolver(g, cfg, precision=prec, ctx=ctx)
        ns.set_state(*st)
        ns.step(0.0)
        torch.cuda.synchronize()
        el, reps = timed_steps(ns_run(ns), args.same_case_steps, stream_of(ctx, ns), flush)
        out[name] = round(world * g.ncell * args.same_case_steps / (max_over_ranks(el, world, device) * 1e-3)
                          / 1e6, 4)
        out[name + "_divergence_max"] = max(r.divergence_max for r in reps)
        out[name + "_poisson_cycles_per_step"] = reps[-1].poisson_iters
        ns.close()
    return out


def batch_key(args, rank, world, local_rank):
    """Both forms on the 96-case batch (config 4) with the default tuning: a
    short run of the batch96 workload, kept as a key of the default line."""
    import copy
    a = copy.copy(args)
    a.steps, a.warmup, a.no_autotune, a.tuning, a.single_form = args.batch_steps, 2, True, None, False
    a.batch, a.batch_seeds, a.precision = 96, None, "mixed"
    d = run_batch(a, rank, world, local_rank)
    return {"workload": d["config"]["workload"], "cells": d["config"]["cells"], "steps": a.steps,
            "forms": d["forms"], "e2e": d["e2e"]["value"], "roofline": d["roofline"],
            "divergence_max": d["divergence_max"], "converged": d["converged"],
            "poisson_iters_mean": d["poisson_iters_mean"], "tuning": "default (no autotune)"}


def large_case(args, ctx, flush, world, device):
    """Both forms on the largest config-3 mesh: the 3-level octree of the
    periodic Taylor-Green box at effective 512^3 (18,712 leaves, 9.58 M leaf
    cells), stepped from the Taylor-Green state with dt from the CFL condition,
    MG-PCG to 1e-10; and the dominant kernel family's roofline on it (direct-
    launch profiled step), where every level has thousands of bricks."""
    import torch

    from nabla_b200 import abi, amr, cases, workloads
    base = args.large_base
    geom, leaves = workloads.tgv_octree(base)
    mesh = amr.AmrMesh(geom, leaves, ctx=ctx)
    cfg = cases.flow_config(reynolds=1600.0, ref_length=1.0, velocity_scale=1.0, cfl=0.4,
                            convection=abi.CONV_WENO5, poisson_tol=1e-10, poisson_max_iters=200)
    hbm, peak_kind = peaks()
    what = "the largest config-3 mesh" if base == 128 else f"base {base}^3"
    out = {"workload": f"3-level octree of the periodic Taylor-Green box at effective {4 * base}^3 ({what}), "
                       "nu=1/1600, WENO-5, CFL 0.4, MG-PCG to 1e-10, from the Taylor-Green state",
           "cells": mesh.ncell, "steps": args.large_steps}
    for name, prec in (("mixed", abi.PRECISION_MIXED), ("fp64", abi.PRECISION_FP64)):
        case = amr.AmrCase(mesh, cfg, precision=prec)
        case.set_state(*workloads.tgv_face_state(case))
        run = ns_run(case)
        run.step()
        torch.cuda.synchronize()
        el, reps = timed_steps(run, args.large_steps, stream_of(ctx, case), flush)
        out[name] = round(world * mesh.ncell * args.large_steps / (max_over_ranks(el, world, device) * 1e-3) / 1e6,
                          4)
        out[name + "_ms_per_step"] = round(el / args.large_steps, 3)
        out[name + "_divergence_max"] = max(r.divergence_max for r in reps)
        out[name + "_poisson_cycles_per_step"] = reps[-1].poisson_iters
        out[name + "_device_bytes"] = int(ctx.lib.nb_case_device_bytes(case.h))
        shares = {fam: profile_step(ctx, run, fam) for fam in FAMILIES}
        shares = {k: v for k, v in shares.items() if v[1] > 0}
        total = sum(v[0] for v in shares.values()) or 1.0
        out[name + "_kernel_shares"] = {k: {"share": round(v[0] / total, 4), "launches": int(v[1]),
                                            "us_per_launch": round(v[0] * 1e3 / v[1], 2)}
                                        for k, v in sorted(shares.items(), key=lambda kv: -kv[1][0])}
        top = max(shares, key=lambda k: shares[k][0])
        ms, nl, nb = shares[top]
        ach = nb / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        out[name + "_roofline"] = {"kernel": top, "bound": "hbm", "achieved": round(ach, 2), "peak": hbm,
                                   "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / hbm, 4),
                                   "launches": int(nl), "avg_launch_us": round(ms * 1e3 / max(nl, 1), 3),
                                   "bytes_per_launch": nb / max(nl, 1)}
        case.close()
    out["mixed_over_fp64"] = round(out["mixed"] / out["fp64"], 3)
    mesh.close()
    return out


class ns_run:
    """A uniform NSSolver or an octree case stepped with dt from its CFL condition."""

    def __init__(self, ns):
        self.ns = ns

    def step(self):
        return self.ns.step(0.0)


def other_form_and_accuracy(args, ctx, run, prec, precision, value, stream, flush, world, device):
    """Times the other arithmetic form on the same mesh, then states the mixed
    form's error against the FP64 form after the same steps from the same state."""
    import torch

    from nabla_b200 import abi
    other_prec = abi.PRECISION_FP64 if prec == abi.PRECISION_MIXED else abi.PRECISION_MIXED
    other_name = "fp64" if precision == "mixed" else "mixed"
    other = make_run(args.workload, ctx, other_prec, mesh=run.mesh)
    for _ in range(args.warmup):
        other.step()
    torch.cuda.synchronize()
    el, reps = timed_steps(other, args.steps, stream_of(ctx, other), flush)
    v_other = world * other.cells * args.steps / (max_over_ranks(el, world, device) * 1e-3) / 1e6
    forms = {precision: round(value, 4), other_name: round(v_other, 4)}
    forms["mixed_over_fp64"] = round(forms["mixed"] / forms["fp64"], 4)
    # accuracy: fresh cases from the initial state, the same number of steps
    n = 10
    a = make_run(args.workload, ctx, abi.PRECISION_FP64, mesh=run.mesh)
    b = make_run(args.workload, ctx, abi.PRECISION_MIXED, mesh=run.mesh)
    ra = rb = None
    for _ in range(n):
        ra, rb = a.step(), b.step()
    sa, sb = a.get_state(), b.get_state()
    acc = {"steps": n, "velocity_rel_err": max(rel_err(x, y) for x, y in zip(sb[:3], sa[:3])),
           "pressure_rel_err": rel_err(sb[3], sa[3]), "mixed_divergence_max": rb.divergence_max,
           "fp64_divergence_max": ra.divergence_max,
           "note": "max-norm errors of the mixed form against the FP64 form (same mesh, same steps)"}
    return forms, acc


def stream_of(ctx, run):
    import torch
    return torch.cuda.ExternalStream(ctx.lib.nb_case_stream(run.h))


# ---------------------------------------------------------------------------
# batched workload: 96 independent octree TGV boxes stepped together
# ---------------------------------------------------------------------------
def batch_specs(n, seeds=None):
    from nabla_b200 import workloads
    return [workloads.tgv_box_case(seed) for seed in (seeds if seeds else range(n))]


def make_batch(ctx, prec, specs):
    from nabla_b200 import amr
    runs = []
    for w in specs:
        mesh = amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
        case = amr.AmrCase(mesh, w.config, precision=prec)
        case.set_state(*w.initial_state(case))
        case._mesh_keepalive = mesh
        runs.append(case)
    return runs


def close_batch(batch):
    for c in batch:
        mesh = c._mesh_keepalive
        c.close()
        mesh.close()


def tune_for(ctx, prec, spec, steps=2):
    """Autotunes the context on one case built from `spec` (cache per GPU)."""
    from nabla_b200 import solver
    (case,) = make_batch(ctx, prec, [spec])
    t0 = time.perf_counter()
    rep = solver.autotune(case, steps=steps)
    rep["tune_s"] = round(time.perf_counter() - t0, 1)
    close_batch([case])
    return rep


def time_batch(ctx, batch, args, stream, flush, world, device):
    """Warm-up steps, then args.steps timed batch steps (L2 flushed before each)."""
    import torch

    from nabla_b200 import solver
    t0 = time.perf_counter()
    solver.batch_step(batch, 0.0, max(1, args.warmup))
    warm_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = ctx.launches
    elapsed = 0.0
    reps = None
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = solver.batch_step(batch, 0.0, 1)
        e1.record(stream)
        e1.synchronize()
        elapsed += e0.elapsed_time(e1)
    return dict(elapsed_max=max_over_ranks(elapsed, world, device), launches=ctx.launches - launches0,
                reps=reps, warm_s=warm_s)


def run_batch(args, rank, world, local_rank):
    import torch

    from nabla_b200 import abi, solver

    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    precision = args.precision or "mixed"
    prec = abi.PRECISION_MIXED if precision == "mixed" else abi.PRECISION_FP64
    other = abi.PRECISION_FP64 if prec == abi.PRECISION_MIXED else abi.PRECISION_MIXED
    specs = batch_specs(args.batch, args.batch_seeds)
    largest = max(specs, key=lambda w: len(w.leaves))
    tuning = {}
    if args.tuning:
        ctx.set_tuning(**args.tuning)
        tuning["fixed"] = ctx.tuning
    elif not args.no_autotune:
        tuning[precision] = tune_for(ctx, prec, largest)
    t0 = time.perf_counter()
    batch = make_batch(ctx, prec, specs)
    setup_s = time.perf_counter() - t0
    cells = sum(c.cell_count for c in batch)
    stream = torch.cuda.ExternalStream(ctx.lib.nb_ctx_stream(ctx.h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    with ClockSampler(local_rank) as clk:
        main = time_batch(ctx, batch, args, stream, flush, world, device)
    elapsed_max, launches, reps = main["elapsed_max"], main["launches"], main["reps"]
    value = world * cells * args.steps / (elapsed_max * 1e-3) / 1e6
    # end to end: every case's state from pinned host memory, one batch step, back to host
    pinned = [[torch.from_numpy(a.copy()).pin_memory().numpy() for a in c.get_state()] for c in batch]
    n_e2e = 2
    e2e_ms = 0.0
    for _ in range(n_e2e):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for c, st in zip(batch, pinned):
            c.set_state(*st)
        solver.batch_step(batch, 0.0, 1)
        for c, st in zip(batch, pinned):
            c.get_state(st)  # straight back into the pinned buffers
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_value = world * cells * n_e2e / (max_over_ranks(e2e_ms, world, device) * 1e-3) / 1e6
    nbytes = sum(a.nbytes for st in pinned for a in st)
    del pinned
    # kernel shares and roofline: direct-launch profiled steps of the largest case
    big = max(batch, key=lambda c: c.cell_count)
    shares = {fam: dict(zip(("ms", "launches", "bytes"), profile_step(ctx, big, fam))) for fam in FAMILIES}
    big = None
    div_max = max(r.divergence_max for r in reps)
    converged = all(bool(r.converged) for r in reps)
    close_batch(batch)
    batch = None
    # the other form on the same cases (same seeds), tuned for its precision
    other_name = "fp64" if other == abi.PRECISION_FP64 else "mixed"
    forms = {precision: round(value, 4)}
    if not args.single_form:
        if not args.no_autotune and not args.tuning:
            tuning[other_name] = tune_for(ctx, other, largest)
        batch2 = make_batch(ctx, other, specs)
        sec = time_batch(ctx, batch2, args, stream, flush, world, device)
        forms[other_name] = round(world * cells * args.steps / (sec["elapsed_max"] * 1e-3) / 1e6, 4)
        div_max = max(div_max, max(r.divergence_max for r in sec["reps"]))
        converged = converged and all(bool(r.converged) for r in sec["reps"])
        close_batch(batch2)
        forms["mixed_over_fp64"] = round(forms["mixed"] / forms["fp64"], 3)
    total = sum(v["ms"] for v in shares.values()) or 1.0
    top = max(shares, key=lambda k: shares[k]["ms"])
    ms, nl, nb = shares[top]["ms"], shares[top]["launches"], shares[top]["bytes"]
    hbm, peak_kind = peaks()
    achieved = nb / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    return {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(elapsed_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == abi.PRECISION_FP64 else "f32+f64",
        "data": "synthetic (96 seeded Taylor-Green boxes with seeded obstacles)",
        "config": {"workload": f"batched: {len(specs)} independent octree TGV boxes, base grids in {{16..64}}^3, "
                               "1-3 levels, 0-6 boxes each, nu=1/1600, WENO-5, CFL 0.4, MG-PCG to 1e-10; "
                               "each step of all cases is one CUDA graph launch",
                   "cases": len(specs), "seeds": args.batch_seeds or f"0..{args.batch - 1}",
                   "cells": cells, "precision": precision,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "setup_s": round(setup_s, 1), "first_steps_s": round(main["warm_s"], 1),
                   "autotune": tuning or "off"},
        "forms": forms,
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 5),
                     "case": "largest case of the batch, direct-launch profiled step",
                     "bytes_per_launch": nb / max(nl, 1), "launches": int(nl), "traffic": None},
        "kernel_shares": {k: round(v["ms"] / total, 4) for k, v in sorted(shares.items(), key=lambda kv: -kv[1]["ms"])},
        "divergence_max": div_max,
        "converged": converged,
        "poisson_iters_mean": round(sum(r.poisson_iters for r in reps) / len(reps), 2),
        "clocks": clk.summary(),
    }


# ---------------------------------------------------------------------------
# pressure-solve precision stress: single projections on 3-level octrees
# ---------------------------------------------------------------------------
def run_poisson(args, rank, world, local_rank):
    import numpy as np
    import torch

    from nabla_b200 import abi, amr, solver, workloads
    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    sizes = []
    for base in args.poisson_bases:
        geom, leaves = workloads.tgv_octree(base)
        mesh = amr.AmrMesh(geom, leaves, ctx=ctx)
        b = np.random.default_rng(base).standard_normal(mesh.ncell)
        hx, hy, hz = mesh.cell_size()
        vol = hx * hy * hz
        b -= np.sum(vol * b) / vol.sum()  # zero volume-weighted mean
        out = {"effective": base * 4, "leaf_cells": mesh.ncell}
        sol = {}
        for name, prec in (("fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
            mesh.solve(b, 1e-12, 400, precision=prec)  # hierarchy set-up and warm-up
            t0 = time.perf_counter()
            x, rep = mesh.solve(b, 1e-12, 400, precision=prec)
            wall = time.perf_counter() - t0
            sol[name] = x
            out[name] = {"iterations": rep.iterations, "residual": rep.residual, "converged": rep.converged,
                         "wall_s": round(wall, 4), "mcells_per_s": round(mesh.ncell / wall / 1e6, 3)}
        d = sol["mixed"] - sol["fp64"]
        scale = np.abs(sol["fp64"]).max()
        r = mesh.apply_a(sol["mixed"]) - b
        out["mixed_vs_fp64"] = {"max_pressure_rel_err": float(np.abs(d).max() / scale),
                                "rms_pressure_rel_err": float(np.sqrt(np.mean(d * d)) / scale),
                                "divergence_rel_residual": float(np.sqrt(np.sum(vol * r * r) / np.sum(vol * b * b)))}
        sizes.append(out)
        mesh.close()
    return {"metric": "pressure-solve precision stress (3-level octrees, rhs N(0,1), tol 1e-12)",
            "unit": "iterations / s", "n_gpus": world, "data": "synthetic (seeded N(0,1) right-hand sides)",
            "config": {"workload": "3-level octrees of the periodic TGV box refined where the brick-mean vorticity "
                                   "is in its top fifth; FP32 V-cycle inside FP64 flexible PCG (mixed) vs FP64 "
                                   "MG-PCG; wall time of nb_amr_poisson_solve incl. the host copies of b and x; "
                                   "the FP64 GPU solution is the reference of the mixed errors"},
            "sizes": sizes, "gpu_launches": int(ctx.launches)}


# ---------------------------------------------------------------------------
# serving: open-loop Poisson arrivals through the continuous-batching loop
# ---------------------------------------------------------------------------
def serve_requests(args, seed):
    """Open-loop Poisson arrivals of config-3-sized requests: each a 3-level
    octree of the periodic Taylor-Green box at effective 128^3, 256^3 or 512^3
    (165 k, 821 k or 9.58 M leaf cells, drawn uniformly) stepped for U[min, max]
    SSP-RK3 steps from the Taylor-Green state. Returns (requests, meshes): the
    payloads exist before the clock starts, as a client's case description
    would; one mesh per size is built on first use and shared by its cases."""
    import threading

    import numpy as np

    from nabla_b200 import abi, amr, cases, serving, workloads
    rng = np.random.default_rng(seed)
    arrivals = serving.poisson_arrivals(args.rate, args.serve_seconds, seed)
    bases = [b for b in (32, 64, 128) if b * 4 <= args.max_effective]
    payloads = {b: workloads.tgv_octree(b) for b in bases}
    cfg = cases.flow_config(reynolds=1600.0, ref_length=1.0, velocity_scale=1.0, cfl=0.4,
                            convection=abi.CONV_WENO5, poisson_tol=1e-10, poisson_max_iters=200)
    meshes, lock = {}, threading.Lock()

    def builder(base):
        def build(ctx, precision):
            with lock:
                if base not in meshes:
                    geom, leaves = payloads[base]
                    meshes[base] = amr.AmrMesh(geom, leaves, ctx=ctx)
            case = amr.AmrCase(meshes[base], cfg, precision=precision)
            case.set_state(*workloads.tgv_face_state(case))
            return case
        return build

    reqs = []
    for i, t in enumerate(arrivals):
        base = bases[int(rng.integers(len(bases)))]
        steps = int(rng.integers(args.min_steps, args.max_steps + 1))
        reqs.append(serving.Request(i, float(t), steps, builder(base), len(payloads[base][1]) * 512))
    return reqs, meshes


def serve_once(args, ctx, prec, seed, time_limit):
    from nabla_b200 import serving
    reqs, meshes = serve_requests(args, seed)
    st = serving.Server(ctx, hbm_budget=150e9, precision=prec, slots=args.slots,
                        builders=args.builders).run(reqs, time_limit=time_limit)
    for m in meshes.values():
        m.close()
    s = st.summary()
    s["unfinished"] = s["arrived"] - s["served"] - s["cancelled"]
    return s


def serve_config(args):
    return (f"serving: open-loop Poisson arrivals at {args.rate}/s for {args.serve_seconds} s; each request a 3-level "
            f"octree of the periodic Taylor-Green box at effective 128^3, 256^3 or 512^3 (config-3 meshes, 165 k / "
            f"821 k / 9.58 M leaf cells), {args.min_steps}-{args.max_steps} steps, HBM budget 150 GB, continuous "
            f"batching ({args.slots} slots, each case collected and relaunched on its own completion, cases built on "
            f"{args.builders} host threads); the loop stops {args.serve_grace} s after the last arrival")


def run_serve(args, rank, world, local_rank):
    import torch

    from nabla_b200 import abi, solver
    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    forms = {}
    for name, prec in (("mixed", abi.PRECISION_MIXED), ("fp64", abi.PRECISION_FP64)):
        with ClockSampler(local_rank) as clk:
            s = serve_once(args, ctx, prec, 7 + rank, args.serve_seconds + args.serve_grace)
        s["clocks"] = clk.summary()
        forms[name] = s
    primary = forms[args.precision or "mixed"]
    return {
        "metric": METRIC, "value": round(primary["mcell_steps_per_s"], 4), "unit": UNIT, "n_gpus": world,
        "steps": None, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if (args.precision or "mixed") == "mixed" else "f64",
        "data": "synthetic (seeded Poisson arrivals of Taylor-Green octree requests)",
        "config": {"workload": serve_config(args), "precision": args.precision or "mixed"},
        "latency": {"p50_s": round(primary["p50_latency_s"], 4), "p99_s": round(primary["p99_latency_s"], 4)},
        "forms": {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in v.items() if kk != "clocks"}
                  for k, v in forms.items()},
        "gpu_launches": int(ctx.launches),
        "clocks": forms["mixed"]["clocks"],
    }


# ---------------------------------------------------------------------------
# CPU baselines (the reference's own code, oracle/_ref)
# ---------------------------------------------------------------------------
def reference_case(name):
    """(grid, config, state, dt or None, description) of the reference's CPU run.
    Built from seeded numpy inputs only: the process that times the reference
    never loads this repository's CUDA library."""
    from nabla_b200 import cases, workloads
    if name == "tgv64":
        g, cfg = cases.taylor_green(64)
        return g, cfg, cases.taylor_green_state(g), None, "the same case"
    if name in ("batch96", "serve"):
        g, cfg = cases.taylor_green(64)
        return g, cfg, cases.taylor_green_state(g), None, \
            "the reference NSSolver on the uniform 64^3 TGV box (the reference has no octree or batched path)"
    g, cfg, st = workloads.channel_uniform(0)
    return g, cfg, st, 0.0, "the reference NSSolver on the uniform-fine 256x64x64 version of the case " \
                            "(same seeded boxes and initial field; the reference has no octree MAC step)"


def host_info():
    """CPU model, logical CPUs of the host and CPUs this process may run on."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cpus": usable,
            "build": "reference sources compiled with g++ -O3 -march=x86-64-v3 (AVX2)"}


def cpu_sample(workload_name, steps):
    """The reference's CPU step on this host (oracle/_ref); returns (s/step, cells, sample)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    g, cfg, st, dt, sample = reference_case(workload_name)
    ref = oracle.Reference()
    ns = ref.ns(g, cfg)
    ns.set_state(*st)
    if dt is None:
        dt = ns.compute_dt()
    t0 = time.perf_counter()
    for _ in range(steps):
        ns.step(dt)
    return (time.perf_counter() - t0) / steps, g.ncell, sample


def _ref_worker(q, workload_name, steps):
    s, cells, sample = cpu_sample(workload_name, steps)
    q.put((s, cells, sample))


def run_large(args, rank, world, local_rank):
    """Both forms on the 512^3-effective octree alone (the `large_case` key of
    the default line as its own workload)."""
    import torch

    from nabla_b200 import solver
    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    ctx = solver.Context(local_rank)
    if args.tuning:
        ctx.set_tuning(**args.tuning)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    args.large_steps = args.steps
    lc = large_case(args, ctx, flush, world, device)
    return {"metric": METRIC, "value": lc["mixed"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": 1, "ms_per_step": lc["mixed_ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (analytic Taylor-Green state)",
            "config": {"workload": lc["workload"], "cells": lc["cells"], "tuning": ctx.tuning},
            "forms": {"mixed": lc["mixed"], "fp64": lc["fp64"], "mixed_over_fp64": lc["mixed_over_fp64"]},
            "roofline": lc["mixed_roofline"], "large_case": lc, "gpu_launches": int(ctx.launches)}


def run_reference(args):
    """Reference arm: the reference's serial CPU step run as one independent
    case per host core (it has no threading), aggregate Mcell-steps/s."""
    import multiprocessing as mp
    cores = int(os.environ.get("NB_REF_CORES", min(os.cpu_count() or 1, 16)))
    steps = max(1, min(args.steps, args.cpu_steps))
    ctxm = mp.get_context("spawn")
    q = ctxm.Queue()
    procs = [ctxm.Process(target=_ref_worker, args=(q, args.workload, steps)) for _ in range(cores)]
    t0 = time.perf_counter()
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    wall = time.perf_counter() - t0
    s_per_step = max(r[0] for r in res)
    cells, sample = res[0][1], res[0][2]
    value = cores * cells / s_per_step / 1e6
    return {
        "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(s_per_step * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, "cells": cells, "precision": "fp64", "sample": sample},
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{steps} NSSolver::step per process, {cores} independent processes; {sample}",
                         "host": host_info()},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="channel3", choices=["channel3", "tgv64", "batch96", "serve", "poisson3", "large"])
    ap.add_argument("--poisson-bases", type=int, nargs="+", default=[32, 64, 128],
                    help="poisson3: base grids (effective = 4x)")
    ap.add_argument("--batch", type=int, default=96, help="cases of the batch96 workload")
    ap.add_argument("--no-autotune", action="store_true", help="batch96: default tuning instead of the autotuner")
    ap.add_argument("--batch-seeds", type=int, nargs="+", default=None,
                    help="batch96: build the batch from these case seeds instead of 0..batch-1")
    ap.add_argument("--single-form", action="store_true", help="batch96: time the primary precision only")
    ap.add_argument("--tuning", type=lambda t: {k: int(v) for k, v in (kv.split("=") for kv in t.split(","))},
                    default=None, help="fixed nb_tuning fields, e.g. threads_per_brick=128,mg_ctas_per_sm=9 "
                    "(channel3, tgv64, batch96)")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    ap.add_argument("--serve-seconds", type=float, default=20.0,
                    help="serve (and the default line's serving key, 0 skips it): arrival window")
    ap.add_argument("--serve-grace", type=float, default=10.0, help="serve: seconds the loop runs after the window")
    ap.add_argument("--min-steps", type=int, default=10)
    ap.add_argument("--max-steps", type=int, default=200)
    ap.add_argument("--max-effective", type=int, default=512, help="serve: largest effective request size (128/256/512)")
    ap.add_argument("--slots", type=int, default=8, help="serve: cases in flight at most")
    ap.add_argument("--builders", type=int, default=4, help="serve: host threads that build admitted cases")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="form reported as `value` (default: mixed for channel3, fp64 for tgv64)")
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--batch-steps", type=int, default=3,
                    help="channel3: timed steps of both forms on the 96-case batch (0: skip)")
    ap.add_argument("--large-steps", type=int, default=5,
                    help="channel3: steps of both forms on the 512^3-effective octree (0: skip)")
    ap.add_argument("--large-base", type=int, default=128,
                    help="base grid of that octree (a multiple of 8; effective 4x): 128 is the largest "
                         "config-3 mesh, smaller bases are profiling cases")
    ap.add_argument("--same-case-steps", type=int, default=5,
                    help="channel3: steps of both forms on the reference arm's uniform-fine case (0: skip)")
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
    runner = {"batch96": run_batch, "serve": run_serve, "poisson3": run_poisson,
              "large": run_large}.get(args.workload, run_ours)
    out = runner(args, rank, world, local_rank)
    if rank == 0:
        if args.cpu_steps > 0 and args.workload not in ("poisson3", "large"):
            s, cells, sample = cpu_sample(args.workload, args.cpu_steps)
            out["cpu_baseline"] = {"value": round(cells / s / 1e6, 5), "unit": UNIT, "cores": 1,
                                   "kind": "reference",
                                   "sample": f"{args.cpu_steps} NSSolver::step, 1 thread: {sample}",
                                   "host": host_info()}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
