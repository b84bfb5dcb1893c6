"""Continuous-batching request loop over the C ABI.

Requests arrive open loop (seeded Poisson process); each asks for `steps`
SSP-RK3 steps of a case. The loop admits waiting requests in arrival order
while a slot is free and their estimated device footprint fits the HBM
budget, builds each admitted case on host threads, and launches its first
step as soon as it exists. Every active case has exactly one step in flight
on its own stream (nb_step_async: the cases' cached step graphs run
concurrently on the GPU). The loop polls the steps in flight
(nb_step_ready) and handles each case on its own completion: it collects the
report (nb_step_wait, which then does not block) and relaunches the case at
once, so a slow case never holds back another case's next step and a new
request joins the device work the moment it is built. A case retires after
its last step: its result is read back, its device memory freed and its slot
given to the next waiting request. State stays resident on the device
between steps; nothing is re-uploaded.

A request can be cancelled at any time (Request.cancel()): a waiting request
is dropped from the queue, a case being built is freed when it arrives, and
an active case is retired after the step it has in flight (a step that is
running on the device is never interrupted), without a result. The
reference's job runner has the same rule for its CPU jobs: one FIFO worker,
cancellation between runs (backend/app/jobs.py:50-140, services.py:120-146).

Latency of a request = completion time - arrival time (queueing, set-up and
steps included), measured on the host clock; throughput = leaf cells x steps
served per second of loop time; offered load = leaf cells x steps of every
request that arrived, per second of the arrival window.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import abi, solver

# device bytes per leaf cell (faces x2 + stage start, pressure, rhs, MG levels,
# PCG vectors), used before a case exists; replaced by the measured footprint
BYTES_PER_CELL = {abi.PRECISION_FP64: 420, abi.PRECISION_MIXED: 380}


@dataclass
class Request:
    rid: int
    arrival: float      # seconds after the start of the loop
    steps: int
    build: object       # callable(ctx, precision) -> case (with .cell_count, .close())
    cells_hint: int     # leaf cells, for admission before the case exists
    done: float = -1.0
    admitted: float = -1.0
    result: object = None
    report: object = None
    cells: int = 0
    steps_done: int = 0
    status: str = "waiting"  # waiting, building, active, done, cancelled
    cancel_requested: bool = False

    def cancel(self):
        """Asks the loop to drop this request (see the module notes for when it takes effect)."""
        self.cancel_requested = True


@dataclass
class ServeStats:
    served: int = 0
    offered: int = 0
    cancelled: int = 0
    arrived: int = 0
    cell_steps: float = 0.0
    offered_cell_steps: float = 0.0
    window_s: float = 0.0
    wall_s: float = 0.0
    latencies: list = field(default_factory=list)
    max_active: int = 0
    max_queue: int = 0
    queue_samples: list = field(default_factory=list)
    peak_bytes: int = 0
    build_s: float = 0.0  # host time spent creating admitted cases
    divergence_max: float = 0.0  # largest post-projection divergence of a served request's last step

    def summary(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        q = np.array(self.queue_samples) if self.queue_samples else np.zeros(1)
        return {"served": self.served, "offered": self.offered, "arrived": self.arrived,
                "cancelled": self.cancelled, "build_s": self.build_s,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mcell_steps_per_s": self.cell_steps / max(self.wall_s, 1e-9) / 1e6, "wall_s": self.wall_s,
                "offered_mcell_steps_per_s": self.offered_cell_steps / max(self.window_s, 1e-9) / 1e6,
                "max_active": self.max_active, "max_queue": self.max_queue,
                "mean_queue": float(q.mean()), "peak_device_bytes": self.peak_bytes,
                "divergence_max": self.divergence_max}


def poisson_arrivals(rate: float, duration: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.array(out)
        out.append(t)


class Server:
    """`slots` caps the cases in flight (continuous batching admits a waiting
    request only when a slot and its footprint are free, so requests finish
    at the rate the device serves them instead of all slowing down together).
    Admitted cases are built on `builders` host threads (ctypes releases the
    GIL; case creation synchronises only its own uploads), so the loop keeps
    collecting and relaunching the active cases while new ones are set up.
    `on_step(request)` (optional) is called after each collected step."""

    def __init__(self, ctx: solver.Context, hbm_budget: float, precision: int = abi.PRECISION_MIXED,
                 keep_results: bool = False, slots: int = 32, builders: int = 2, poll_s: float = 2e-4,
                 on_step=None):
        self.ctx, self.budget, self.precision, self.keep = ctx, hbm_budget, precision, keep_results
        self.slots, self.builders, self.poll_s, self.on_step = slots, builders, poll_s, on_step

    def _build(self, r: Request):
        b0 = time.perf_counter()
        case = r.build(self.ctx, self.precision)
        return case, time.perf_counter() - b0

    def run(self, requests: list[Request], time_limit: float | None = None) -> ServeStats:
        from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
        st = ServeStats(offered=len(requests))
        pending = sorted(requests, key=lambda r: r.arrival)
        st.window_s = max((r.arrival for r in pending), default=0.0)
        queue: list[Request] = []
        active: list[tuple[Request, object]] = []          # each with one step in flight
        building: list[tuple[Request, object, float]] = []  # (request, future, reserved bytes)
        used = 0.0
        t0 = time.perf_counter()
        nxt = 0
        pool = ThreadPoolExecutor(max_workers=max(1, self.builders))

        def retire(r, case, status):
            nonlocal used
            r.status = status
            r.done = time.perf_counter() - t0
            used -= self.ctx.lib.nb_case_device_bytes(case.h)
            case.close()

        try:
            while nxt < len(pending) or queue or active or building:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit:
                    break
                while nxt < len(pending) and pending[nxt].arrival <= now:
                    r = pending[nxt]
                    st.arrived += 1
                    st.offered_cell_steps += r.cells_hint * r.steps
                    queue.append(r)
                    nxt += 1
                for r in [r for r in queue if r.cancel_requested]:
                    queue.remove(r)
                    r.status = "cancelled"
                    st.cancelled += 1
                st.max_queue = max(st.max_queue, len(queue))
                st.queue_samples.append(len(queue))
                # admission: arrival order, slots, HBM budget (the first case always fits)
                while queue and len(active) + len(building) < self.slots:
                    r = queue[0]
                    need = r.cells_hint * BYTES_PER_CELL[self.precision]
                    if (active or building) and used + need > self.budget:
                        break
                    queue.pop(0)
                    r.admitted = time.perf_counter() - t0
                    r.status = "building"
                    used += need
                    building.append((r, pool.submit(self._build, r), need))
                progressed = False
                still_building = []
                for r, fut, need in building:
                    if not fut.done():
                        still_building.append((r, fut, need))
                        continue
                    case, dt = fut.result()
                    st.build_s += dt
                    r.cells = case.cell_count
                    used += self.ctx.lib.nb_case_device_bytes(case.h) - need
                    progressed = True
                    if r.cancel_requested:
                        retire(r, case, "cancelled")
                        st.cancelled += 1
                        continue
                    r.status = "active"
                    solver.step_async(case, 0.0)
                    active.append((r, case))
                building = still_building
                st.max_active = max(st.max_active, len(active) + len(building))
                st.peak_bytes = max(st.peak_bytes, used)
                # collect every case whose own step has finished, relaunch it at once
                still = []
                for r, case in active:
                    if not solver.step_ready(case):
                        still.append((r, case))
                        continue
                    progressed = True
                    rep = solver.step_wait(case)
                    r.steps_done += 1
                    st.cell_steps += r.cells
                    if self.on_step is not None:
                        self.on_step(r)
                    if r.cancel_requested:
                        retire(r, case, "cancelled")
                        st.cancelled += 1
                    elif r.steps_done >= r.steps:
                        r.report = rep
                        st.divergence_max = max(st.divergence_max, rep.divergence_max)
                        if self.keep:
                            r.result = case.get_state()
                        retire(r, case, "done")
                        st.served += 1
                        st.latencies.append(r.done - r.arrival)
                    else:
                        solver.step_async(case, 0.0)
                        still.append((r, case))
                active = still
                if progressed:
                    continue
                if active:
                    time.sleep(self.poll_s)
                elif building:
                    wait([f for _, f, _ in building], timeout=0.05, return_when=FIRST_COMPLETED)
                elif nxt < len(pending) and not queue:
                    time.sleep(max(0.0, min(0.05, pending[nxt].arrival - (time.perf_counter() - t0))))
            st.wall_s = time.perf_counter() - t0
        finally:
            for _, case in active:
                case.close()
            for _, fut, _ in building:
                case, _ = fut.result()
                case.close()
            pool.shutdown(wait=True)
        return st
