"""Continuous-batching request loop over the C ABI.

Requests arrive open loop (seeded Poisson process); each asks for `steps`
SSP-RK3 steps of a case. The loop admits waiting requests in arrival order
while their estimated device footprint fits the HBM budget, builds each
admitted case on the device, and then, every iteration, launches one step of
every active case on its own stream (nb_step_async: the cases' cached step
graphs run concurrently on the GPU) and collects them (nb_step_wait). A case
retires after its last step: its result is read back, its device memory
freed, and its slot given to the next waiting request. State stays resident
on the device between steps; nothing is re-uploaded.

Latency of a request = completion time - arrival time (queueing, set-up and
steps included), measured on the host clock; throughput = leaf cells x steps
served per second of loop time.
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


@dataclass
class ServeStats:
    served: int = 0
    offered: int = 0
    cell_steps: float = 0.0
    wall_s: float = 0.0
    latencies: list = field(default_factory=list)
    max_active: int = 0
    max_queue: int = 0
    peak_bytes: int = 0
    build_s: float = 0.0  # host time spent creating admitted cases

    def summary(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        return {"served": self.served, "offered": self.offered, "build_s": self.build_s,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mcell_steps_per_s": self.cell_steps / max(self.wall_s, 1e-9) / 1e6, "wall_s": self.wall_s,
                "max_active": self.max_active, "max_queue": self.max_queue, "peak_device_bytes": self.peak_bytes}


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
    launching steps of the active cases while new ones are set up."""

    def __init__(self, ctx: solver.Context, hbm_budget: float, precision: int = abi.PRECISION_MIXED,
                 keep_results: bool = False, slots: int = 32, builders: int = 2):
        self.ctx, self.budget, self.precision, self.keep = ctx, hbm_budget, precision, keep_results
        self.slots, self.builders = slots, builders

    def _build(self, r: Request):
        b0 = time.perf_counter()
        case = r.build(self.ctx, self.precision)
        return case, time.perf_counter() - b0

    def run(self, requests: list[Request], time_limit: float | None = None) -> ServeStats:
        from concurrent.futures import ThreadPoolExecutor, wait, FIRST_COMPLETED
        st = ServeStats(offered=len(requests))
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list[Request] = []
        active: list[tuple[Request, object, int]] = []  # (request, case, steps left)
        building: list[tuple[Request, object, float]] = []  # (request, future, reserved bytes)
        used = 0.0
        t0 = time.perf_counter()
        nxt = 0
        pool = ThreadPoolExecutor(max_workers=max(1, self.builders))
        try:
            while nxt < len(pending) or queue or active or building:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit:
                    break
                while nxt < len(pending) and pending[nxt].arrival <= now:
                    queue.append(pending[nxt])
                    nxt += 1
                st.max_queue = max(st.max_queue, len(queue))
                # launch one step of every active case; admit and build while they run
                for _, case, _ in active:
                    solver.step_async(case, 0.0)
                while queue and len(active) + len(building) < self.slots:
                    r = queue[0]
                    need = r.cells_hint * BYTES_PER_CELL[self.precision]
                    if (active or building) and used + need > self.budget:
                        break
                    queue.pop(0)
                    r.admitted = time.perf_counter() - t0
                    used += need
                    building.append((r, pool.submit(self._build, r), need))
                joined, still_building = [], []
                for r, fut, need in building:
                    if not fut.done():
                        still_building.append((r, fut, need))
                        continue
                    case, dt = fut.result()
                    st.build_s += dt
                    r.cells = case.cell_count
                    used += self.ctx.lib.nb_case_device_bytes(case.h) - need
                    joined.append((r, case, r.steps))
                building = still_building
                st.max_active = max(st.max_active, len(active) + len(joined) + len(building))
                st.peak_bytes = max(st.peak_bytes, used)
                if not active:
                    active = joined
                    if not active:
                        if building:
                            wait([f for _, f, _ in building], timeout=0.05, return_when=FIRST_COMPLETED)
                        elif nxt < len(pending):
                            time.sleep(max(0.0, pending[nxt].arrival - (time.perf_counter() - t0)))
                    continue
                still = []
                for r, case, left in active:
                    rep = solver.step_wait(case)
                    st.cell_steps += r.cells
                    left -= 1
                    if left > 0:
                        still.append((r, case, left))
                        continue
                    r.done = time.perf_counter() - t0
                    r.report = rep
                    if self.keep:
                        r.result = case.get_state()
                    st.served += 1
                    st.latencies.append(r.done - r.arrival)
                    used -= self.ctx.lib.nb_case_device_bytes(case.h)
                    case.close()
                active = still + joined
            st.wall_s = time.perf_counter() - t0
        finally:
            for _, case, _ in active:
                case.close()
            for _, fut, _ in building:
                case, _ = fut.result()
                case.close()
            pool.shutdown(wait=True)
        return st
