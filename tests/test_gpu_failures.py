"""Failure handling through the public API, made on the host.

* A NaN planted in a case's input state is reported as NB_ERR_NAN by the
  step (the reference's per-step acceptance gate rejects a non-finite step,
  core/src/flow/ns_solver.cpp:797-823), on uniform and octree cases and on
  the asynchronous path, and the context stays usable afterwards.
* A Poisson cycle cap too small to converge is a status in the reports, not
  an error (PoissonSolver::Report::converged, core/include/nabla/flow/
  poisson.hpp:24-28): the step returns NB_OK with converged = 0.
* A request cancelled while its case is on the device (and one cancelled
  while it waits) is retired by the serving loop without a result, and the
  other requests' results are unchanged.

No device fault is provoked: every device loop is bounded by its cycle cap.
"""
import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, serving, solver, workloads

pytestmark = pytest.mark.gpu


def _tgv16(ctx, poison=None, max_iters=None):
    g, cfg = cases.taylor_green(16)
    if max_iters is not None:
        cfg.poisson_max_iters = max_iters
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    st = [np.array(a, copy=True) for a in cases.taylor_green_state(g)]
    if poison is not None:
        st[poison[0]][poison[1]] = np.nan
    ns.set_state(*st)
    return ns


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_nan_in_uniform_state_is_reported(ctx, precision):
    g, cfg = cases.taylor_green(16)
    ns = solver.NSSolver(g, cfg, precision=precision, ctx=ctx)
    st = [np.array(a, copy=True) for a in cases.taylor_green_state(g)]
    st[0][123] = np.nan
    ns.set_state(*st)
    with pytest.raises(solver.NablaError) as e:
        ns.step(0.05)
    assert e.value.status == abi.NB_ERR_NAN
    ns.close()
    # the context is still usable: a clean case steps and converges
    ok = _tgv16(ctx)
    r = ok.step(0.05)
    assert r.converged and r.divergence_max < 1e-8
    ok.close()


def test_nan_in_octree_state_is_reported_sync_and_async(ctx):
    w = workloads.tgv_box_case(0)
    mesh = amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
    case = amr.AmrCase(mesh, w.config)
    st = [np.array(a, copy=True) for a in w.initial_state(case)]
    st[1][len(st[1]) // 3] = np.nan
    case.set_state(*st)
    with pytest.raises(solver.NablaError) as e:
        case.step(0.01)
    assert e.value.status == abi.NB_ERR_NAN
    case.set_state(*st)
    solver.step_async(case, 0.01)
    with pytest.raises(solver.NablaError) as e:
        solver.step_wait(case)
    assert e.value.status == abi.NB_ERR_NAN
    case.close()
    mesh.close()


def test_cycle_cap_reports_non_convergence_as_status(ctx):
    ns = _tgv16(ctx, max_iters=1)
    r = ns.step(0.05)  # NB_OK: no exception
    assert r.converged == 0 and r.poisson_iters <= 3
    ns.close()
    g, _ = cases.taylor_green(16)
    b = np.random.default_rng(1).standard_normal(g.ncell)
    b -= b.mean()
    x, rep = solver.MgPoisson(1e-12, 1, ctx=ctx).solve(g, b)
    assert not rep.converged and rep.iterations == 1


def test_cancel_queued_and_in_flight_requests(ctx):
    from test_gpu_serving import _builder, _small_seeds
    seeds = _small_seeds(4)
    cells = [len(workloads.tgv_box_case(s).leaves) * 512 for s in seeds]
    reqs = [serving.Request(i, 0.0, 6, _builder(s), cells[i]) for i, s in enumerate(seeds)]

    def on_step(r):
        if r.rid == 1 and r.steps_done == 2:
            r.cancel()        # in flight: retired after this step
            reqs[3].cancel()  # still waiting for a slot

    srv = serving.Server(ctx, hbm_budget=4e9, precision=abi.PRECISION_FP64, keep_results=True, slots=2,
                         on_step=on_step)
    stats = srv.run(reqs)
    assert reqs[1].status == "cancelled" and reqs[1].steps_done == 2 and reqs[1].result is None
    assert reqs[3].status == "cancelled" and reqs[3].steps_done == 0
    assert stats.served == 2 and stats.cancelled == 2
    for r in (reqs[0], reqs[2]):
        assert r.status == "done"
        case = r.build(ctx, abi.PRECISION_FP64)
        for _ in range(r.steps):
            case.step()
        for x, y in zip(r.result, case.get_state()):
            assert np.array_equal(x, y)
        case.close()
