"""Outer iterative refinement of the mixed form: the FP64 flexible PCG with
the FP32 V-cycle stops on its recursively updated residual, then the FP64
true residual rhs - A x decides; above the tolerance the solve restarts from
x with that residual (at most twice). The solve reports the true residual,
so a converged mixed solve meets the tolerance on the true residual, and
its pressure matches the FP64 form's (the same operator) at the tolerance's
level. Both the host-driven solve (nb_poisson_solve) and the graph-captured
step exercise it; a projection that needs no restart is unchanged."""
import numpy as np
import pytest

from helpers import channel_block_grid, rel_err
from nabla_b200 import abi, cases, solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tol", [1e-10, 1e-12, 1e-13])
def test_mixed_solve_meets_tolerance_on_true_residual(ctx, tol):
    g = channel_block_grid()
    b = np.random.default_rng(2024).standard_normal(g.ncell)
    x, rep = solver.MgPoisson(tol, 300, precision=abi.PRECISION_MIXED, ctx=ctx).solve(g, b)
    assert rep.converged
    assert rep.residual <= tol
    xd, rd = solver.MgPoisson(tol, 300, precision=abi.PRECISION_FP64, ctx=ctx).solve(g, b)
    assert rel_err(x, xd) < max(1e-6, 1e4 * tol)


@pytest.mark.parametrize("tol", [1e-11, 1e-13])
def test_periodic_mixed_solve_meets_tolerance(ctx, tol):
    g, _ = cases.taylor_green(32)
    b = np.random.default_rng(7).standard_normal(g.ncell)
    b -= b.mean()
    x, rep = solver.MgPoisson(tol, 300, precision=abi.PRECISION_MIXED, ctx=ctx).solve(g, b)
    assert rep.converged and rep.residual <= tol


def test_mixed_step_reports_true_residual_within_tolerance(ctx):
    g, cfg = cases.taylor_green(32)
    cfg.poisson_tol = 1e-12
    ns = solver.NSSolver(g, cfg, precision=abi.PRECISION_MIXED, ctx=ctx)
    ns.set_state(*cases.taylor_green_state(g))
    for _ in range(2):
        r = ns.step(0.07)
        assert r.converged and r.poisson_residual <= 1e-12 and r.divergence_max < 1e-8
    ns.close()
