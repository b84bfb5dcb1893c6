"""Continuous-batching request loop (nabla_b200.serving): requests that arrive
while others are on the GPU are admitted as budget frees up and their steps
overlap with the running ones. Each result must be the same alone and in the
mix: served results are compared bit for bit with the same case stepped by
itself."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, serving, solver, workloads

pytestmark = pytest.mark.gpu


def _small_seeds(n):
    out = []
    s = 0
    while len(out) < n:
        w = workloads.tgv_box_case(s)
        if len(w.leaves) * 512 <= 200_000:
            out.append(s)
        s += 1
    return out


def _builder(seed):
    def build(ctx, precision):
        w = workloads.tgv_box_case(seed)
        mesh = amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
        case = amr.AmrCase(mesh, w.config, precision=precision)
        case.set_state(*w.initial_state(case))
        case._mesh_keepalive = mesh
        return case
    return build


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_each_result_is_the_same_alone_and_in_the_mix(ctx, precision):
    seeds = _small_seeds(5)
    steps = [4, 2, 5, 3, 2]
    arrivals = [0.0, 0.0, 0.05, 0.1, 0.12]
    reqs = [serving.Request(i, arrivals[i], steps[i], _builder(s), len(workloads.tgv_box_case(s).leaves) * 512)
            for i, s in enumerate(seeds)]
    srv = serving.Server(ctx, hbm_budget=2e9, precision=precision, keep_results=True)
    stats = srv.run(reqs)
    assert stats.served == len(reqs)
    assert stats.max_active >= 2  # the steps really overlapped
    for r in reqs:
        case = r.build(ctx, precision)
        for _ in range(r.steps):
            rep = case.step()
        for x, y in zip(r.result, case.get_state()):
            assert np.array_equal(x, y)
        assert rep.divergence_max == r.report.divergence_max
        assert r.report.converged and r.report.divergence_max < 1e-8
        case.close()
    s = stats.summary()
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0.0


def test_budget_limits_admission(ctx):
    seeds = _small_seeds(3)
    reqs = [serving.Request(i, 0.0, 2, _builder(s), len(workloads.tgv_box_case(s).leaves) * 512)
            for i, s in enumerate(seeds)]
    # a budget below any single case still serves them, one at a time
    stats = serving.Server(ctx, hbm_budget=1.0, precision=abi.PRECISION_MIXED).run(reqs)
    assert stats.served == 3 and stats.max_active == 1


def test_async_step_rules(ctx):
    case = _builder(_small_seeds(1)[0])(ctx, abi.PRECISION_FP64)
    solver.step_async(case)
    with pytest.raises(solver.NablaError):
        solver.step_async(case)
    with pytest.raises(solver.NablaError):
        case.step()
    rep = solver.step_wait(case)
    assert rep.converged
    with pytest.raises(solver.NablaError):
        solver.step_wait(case)
    case.close()
