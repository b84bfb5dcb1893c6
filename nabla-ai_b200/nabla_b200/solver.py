"""Host-side mirror of the reference's solver seams over the C ABI.

Same names, argument meaning and error behaviour as the reference:

* ``MgPoisson(tol, max_cycles).solve(grid, b) -> (x, Report)`` —
  ``nabla::flow::MgPoisson`` / ``PoissonSolver::solve``
  (core/include/nabla/flow/poisson.hpp:20-33, :77-91).
* ``apply_a(grid, x)`` — ``CgPoisson::applyA`` (core/src/flow/poisson.cpp:102-134).
* ``NSSolver(grid, config)`` with ``initialize / step / set_state / u_face ...``
  — ``nabla::flow::NSSolver`` (core/include/nabla/flow/ns_solver.hpp:58-156).

Errors raise ``NablaError`` (the reference throws std::runtime_error); solver
non-convergence is reported in ``Report.converged`` and is not an error.
Every call runs on the CUDA library; nothing here computes the solution.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import abi
from .cases import Grid


class NablaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


@dataclass
class Report:
    iterations: int
    residual: float
    converged: bool


class Context:
    """One CUDA device. ``Context(device)`` fails loudly without an sm_100 GPU."""

    def __init__(self, device: int = 0):
        self.lib = abi.load()
        h = C.c_void_p()
        st = self.lib.nb_ctx_create(device, C.byref(h))
        if st != abi.NB_OK:
            raise NablaError(st, "nb_ctx_create failed: " + self.lib.nb_status_string(st).decode())
        self.h = h

    def check(self, st: int, what: str):
        if st != abi.NB_OK:
            raise NablaError(st, f"{what}: {self.lib.nb_last_error(self.h).decode()}")

    @property
    def launches(self) -> int:
        return self.lib.nb_ctx_launch_count(self.h)

    @property
    def tuning(self) -> dict:
        """The nb_tuning applied to cases, meshes and Poisson hierarchies created next."""
        t = abi.Tuning()
        self.check(self.lib.nb_ctx_get_tuning(self.h, C.byref(t)), "nb_ctx_get_tuning")
        return t.as_dict()

    def set_tuning(self, **fields):
        """Sets nb_tuning fields (the others keep their current values)."""
        t = abi.Tuning()
        self.check(self.lib.nb_ctx_get_tuning(self.h, C.byref(t)), "nb_ctx_get_tuning")
        for k, v in fields.items():
            if k not in t.as_dict():
                raise ValueError(f"unknown tuning field {k!r}")
            setattr(t, k, int(v))
        self.check(self.lib.nb_ctx_set_tuning(self.h, C.byref(t)), "nb_ctx_set_tuning")

    def close(self):
        if getattr(self, "h", None):
            self.lib.nb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def apply_a(grid: Grid, x: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    ctx = ctx or default_context()
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(grid.ncell)
    ctx.check(ctx.lib.nb_apply_laplacian(ctx.h, C.byref(grid.desc()), abi.dptr(x), abi.dptr(out)),
              "nb_apply_laplacian")
    return out


class MgPoisson:
    """Geometric-multigrid-preconditioned flexible CG on the GPU."""

    def __init__(self, tol: float = 1e-9, max_cycles: int = 100, precision: int = abi.PRECISION_FP64,
                 ctx: Context | None = None):
        self.tol, self.max_cycles, self.precision = tol, max_cycles, precision
        self.ctx = ctx or default_context()

    def name(self) -> str:
        return "mg-pcg" if self.precision == abi.PRECISION_FP64 else "mg-pcg-mixed"

    def solve(self, grid: Grid, b: np.ndarray):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(grid.ncell)
        rep = abi.PoissonReport()
        self.ctx.check(self.ctx.lib.nb_poisson_solve(self.ctx.h, C.byref(grid.desc()), abi.dptr(b),
                                                     abi.dptr(x), self.tol, self.max_cycles,
                                                     self.precision, C.byref(rep)),
                       "nb_poisson_solve")
        return x, Report(rep.iterations, rep.residual, bool(rep.converged))


class NSSolver:
    """Staggered SSP-RK3 / WENO-5 / MG-PCG step, state resident on the device."""

    def __init__(self, grid: Grid, config: abi.FlowConfig, precision: int = abi.PRECISION_FP64,
                 ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.grid, self.config = grid, config
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.nb_case_create(self.ctx.h, C.byref(grid.desc()), C.byref(config),
                                                   precision, C.byref(h)), "nb_case_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.nb_case_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def initialize(self):
        self.ctx.check(self.ctx.lib.nb_case_initialize(self.h), "initialize")

    def sample(self, component: int, points) -> np.ndarray:
        """SolverBackend::sample for many points: component 0-2 = cell-centred
        velocity of the containing cell, 3 = its pressure (nb_case_sample)."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(pts.shape[0])
        self.ctx.check(self.ctx.lib.nb_case_sample(self.h, component, pts.shape[0], abi.dptr(pts), abi.dptr(out)),
                       "nb_case_sample")
        return out

    def write_vtu(self, path):
        """VTK XML unstructured grid of the cell-centred state (nb_case_write_vtu)."""
        self.ctx.check(self.ctx.lib.nb_case_write_vtu(self.h, str(path).encode()), "write_vtu")

    def write_checkpoint(self, path):
        """writeCheckpoint (core/src/flow/case.cpp:274-294): the reference's NBFCK01 file."""
        self.ctx.check(self.ctx.lib.nb_case_write_checkpoint(self.h, str(path).encode()), "write_checkpoint")

    def read_checkpoint(self, path):
        """readCheckpoint (core/src/flow/case.cpp:296-319): state and step clock from an NBFCK01 file."""
        self.ctx.check(self.ctx.lib.nb_case_read_checkpoint(self.h, str(path).encode()), "read_checkpoint")

    def set_state(self, u, v, w, p, step=0, t=0.0, dt_last=0.0):
        nu, nv, nw, np_ = self.grid.sizes()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, p)]
        if [a.size for a in arrs] != [nu, nv, nw, np_]:
            raise NablaError(abi.NB_ERR_BAD_ARG, "NSSolver::setState: size mismatch")
        self.ctx.check(self.ctx.lib.nb_case_set_state(self.h, *[abi.dptr(a) for a in arrs], step, t,
                                                      dt_last), "setState")

    def get_state(self, out=None):
        """u, v, w, p in the reference's MAC layout. `out`: four contiguous
        float64 arrays of the right sizes to copy into (pinned buffers make
        the read-back one DMA per array, no host copy)."""
        sizes = list(self.grid.sizes())
        if out is None:
            out = [np.zeros(n) for n in sizes]
        elif [a.size for a in out] != sizes or not all(
                a.dtype == np.float64 and a.flags.c_contiguous and a.flags.writeable for a in out):
            raise NablaError(abi.NB_ERR_BAD_ARG, "get_state: out must be four writeable contiguous float64 arrays "
                                                 "of the state sizes")
        u, v, w, p = out
        self.ctx.check(self.ctx.lib.nb_case_get_state(self.h, abi.dptr(u), abi.dptr(v), abi.dptr(w),
                                                      abi.dptr(p)), "get_state")
        return u, v, w, p

    def u_face(self):
        return self.get_state()[0]

    def pressure(self):
        return self.get_state()[3]

    def clock(self):
        st, t, dt = C.c_int(), C.c_double(), C.c_double()
        self.ctx.check(self.ctx.lib.nb_case_get_clock(self.h, C.byref(st), C.byref(t), C.byref(dt)),
                       "clock")
        return st.value, t.value, dt.value

    def compute_dt(self) -> float:
        dt = C.c_double()
        self.ctx.check(self.ctx.lib.nb_case_compute_dt(self.h, C.byref(dt)), "computeDt")
        return dt.value

    def step(self, dt: float = 0.0) -> abi.StepReport:
        rep = abi.StepReport()
        self.ctx.check(self.ctx.lib.nb_step(self.h, dt, C.byref(rep)), "step")
        return rep

    def step_many(self, dt: float, n: int) -> abi.StepReport:
        rep = abi.StepReport()
        self.ctx.check(self.ctx.lib.nb_step_many(self.h, dt, n, C.byref(rep)), "step_many")
        return rep

    @property
    def device_bytes(self) -> int:
        return self.ctx.lib.nb_case_device_bytes(self.h)

    @property
    def cell_count(self) -> int:
        return self.ctx.lib.nb_case_cell_count(self.h)


def batch_step(cases, dt: float = 0.0, nsteps: int = 1):
    """Steps independent cases (NSSolver or amr.AmrCase objects of one
    context) together: each step of all of them is one CUDA graph launch
    (nb_batch_step). Returns each case's last StepReport."""
    cases = list(cases)
    if not cases:
        return []
    ctx = cases[0].ctx
    if any(c.ctx is not ctx for c in cases):
        raise ValueError("batch cases must share one context")
    hs = (C.c_void_p * len(cases))(*[c.h.value if isinstance(c.h, C.c_void_p) else c.h for c in cases])
    reps = (abi.StepReport * len(cases))()
    ctx.check(ctx.lib.nb_batch_step(ctx.h, hs, len(cases), dt, nsteps, reps), "nb_batch_step")
    return list(reps)


def step_async(case, dt: float = 0.0):
    """Launches one step of `case` (NSSolver or amr.AmrCase) without waiting."""
    case.ctx.check(case.ctx.lib.nb_step_async(case.h, dt), "nb_step_async")


def step_wait(case) -> abi.StepReport:
    """Waits for the step launched by step_async and returns its report."""
    rep = abi.StepReport()
    case.ctx.check(case.ctx.lib.nb_step_wait(case.h, C.byref(rep)), "nb_step_wait")
    return rep


def step_ready(case) -> bool:
    """True once the step launched by step_async has finished on the device
    (step_wait then returns without waiting)."""
    r = C.c_int()
    case.ctx.check(case.ctx.lib.nb_step_ready(case.h, C.byref(r)), "nb_step_ready")
    return bool(r.value)


def default_tuning() -> dict:
    t = abi.Tuning()
    abi.load().nb_tuning_default(C.byref(t))
    return t.as_dict()


def default_tune_cache() -> str:
    """Per-user tuning cache: $NABLA_B200_TUNE_CACHE, else
    ~/.cache/nabla_b200/tuning.txt (the directory is created)."""
    path = os.environ.get("NABLA_B200_TUNE_CACHE")
    if not path:
        path = os.path.join(os.path.expanduser("~"), ".cache", "nabla_b200", "tuning.txt")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    return path


def autotune(case, steps: int = 3, cache: str | None = "default") -> dict:
    """nb_autotune on `case` (NSSolver or amr.AmrCase): picks the fastest
    converging tuning for cases like it and sets it on the case's context
    (cases created afterwards use it). cache=None times without a cache;
    "default" uses default_tune_cache()."""
    ctx = case.ctx
    path = default_tune_cache() if cache == "default" else cache
    rep = abi.TuneReport()
    ctx.check(ctx.lib.nb_autotune(ctx.h, case.h, steps, path.encode() if path else None, C.byref(rep)),
              "nb_autotune")
    return {"best": rep.best.as_dict(), "best_ms": rep.best_ms, "default_ms": rep.default_ms,
            "candidates": rep.candidates, "rejected": rep.rejected, "from_cache": bool(rep.from_cache),
            "key": rep.key.decode()}


def checkpoint_info(path) -> dict | None:
    """Header of a checkpoint file (host only): kind "uniform" (NBFCK01, dims)
    or "octree" (NBFAMR1, leaf count), step, t, dt; None if unreadable."""
    kind, dims = C.c_int32(), (C.c_int32 * 3)()
    nleaf, step, t, dt = C.c_int64(), C.c_int32(), C.c_double(), C.c_double()
    if abi.load().nb_checkpoint_info(str(path).encode(), C.byref(kind), dims, C.byref(nleaf), C.byref(step),
                                     C.byref(t), C.byref(dt)) != 0:
        return None
    out = {"kind": "uniform" if kind.value == 0 else "octree", "step": step.value, "t": t.value, "dt": dt.value}
    if kind.value == 0:
        out["dims"] = tuple(dims)
    else:
        out["leaves"] = nleaf.value
    return out


def run_case(grid: Grid, config: abi.FlowConfig, run_dir, max_steps: int, *, checkpoint_every: int = 0,
             snapshot_every: int = 0, stop_time: float = 0.0, steady_tol: float = 0.0, restart_from=None,
             precision: int = abi.PRECISION_FP64, ctx: Context | None = None) -> dict:
    """nb_run_case: runCase (core/src/flow/case.cpp:349-401) on the GPU, writing
    diagnostics.jsonl and checkpoints into run_dir. Returns the RunSummary."""
    ctx = ctx or default_context()
    opt = abi.RunOptions(str(run_dir).encode(), max_steps, checkpoint_every, stop_time, steady_tol,
                         str(restart_from).encode() if restart_from else None, precision, snapshot_every)
    out = abi.RunSummary()
    ctx.check(ctx.lib.nb_run_case(ctx.h, C.byref(grid.desc()), C.byref(config), C.byref(opt), C.byref(out)),
              "nb_run_case")
    return out.as_dict()


def load_case(path) -> dict:
    """loadCase (core/src/flow/case.cpp:136-170) for a case JSON file: the same
    keys, case types, builder defaults and run options, plus this library's keys
    "precision" ("fp64" default, or "mixed") and "backend" ("cuda"; "cpu" names the
    reference's own solver and is refused here). Returns name, grid, config, run
    (run_case keyword arguments), precision and backend."""
    import json

    from . import cases
    j = json.loads(open(path).read())
    kind = j.get("type", "lid-cavity")
    re_, res = float(j.get("reynolds", 100.0)), int(j.get("resolution", 64))
    run = dict(max_steps=20000, snapshot_every=0, checkpoint_every=0, stop_time=0.0, steady_tol=0.0)
    if kind == "lid-cavity":
        grid, cfg = cases.lid_cavity(res, re_, float(j.get("lid_velocity", 1.0)))
        run.update(max_steps=60000, steady_tol=1e-6)
    elif kind in ("channel", "poiseuille"):
        grid, cfg = cases.channel(int(j.get("nx", 6 * res)), res, re_, float(j.get("bulk_velocity", 1.0)))
        run.update(max_steps=40000, steady_tol=1e-6)
    elif kind == "wall-mounted-cube":
        grid, cfg = cases.wall_mounted_cube(res, re_)
        run.update(max_steps=200, snapshot_every=50, checkpoint_every=50)
    else:
        raise ValueError(f"loadCase: unknown case type '{kind}'")
    cfg.cfl = float(j.get("cfl", cfg.cfl))
    if j.get("convection") == "weno5":
        cfg.convection = abi.CONV_WENO5
    elif j.get("convection") == "central":
        cfg.convection = abi.CONV_CENTRAL
    run["run_dir"] = j.get("run_dir", "run_" + kind)
    for key, cast in (("max_steps", int), ("snapshot_every", int), ("checkpoint_every", int),
                      ("stop_time", float), ("steady_tol", float)):
        if key in j:
            run[key] = cast(j[key])
    run["restart_from"] = j.get("restart_from") or None
    backend = j.get("backend", "cuda")
    if backend != "cuda":
        raise ValueError(f"load_case: backend '{backend}' is not this library's (use \"cuda\")")
    precision = {"fp64": abi.PRECISION_FP64, "mixed": abi.PRECISION_MIXED}.get(j.get("precision", "fp64"))
    if precision is None:
        raise ValueError(f"load_case: unknown precision '{j.get('precision')}'")
    return dict(name=j.get("name", kind), grid=grid, config=cfg, run=run, precision=precision, backend=backend)


def run_case_file(path, ctx: Context | None = None) -> dict:
    """`nabla_solve run <case.json>` on the GPU: load_case + run_case."""
    spec = load_case(path)
    run = dict(spec["run"])
    run_dir = run.pop("run_dir")
    max_steps = run.pop("max_steps")
    return run_case(spec["grid"], spec["config"], run_dir, max_steps, precision=spec["precision"], ctx=ctx, **run)
