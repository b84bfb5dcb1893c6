"""Grid-resident V-cycle (nb_tuning.vgrid, off by default): every V-cycle is one
cooperative launch whose CTAs run the phases (sweeps, residual + restriction,
coarsest solve, prolongation) of all levels with a bounded grid barrier
between them. Each phase is the per-sweep launch path's own per-brick code,
so the per-cell arithmetic is the same; only the order of grid-wide sums
(pending means, the PCG dots) differs. Checked against the per-sweep form:
FP64 within 1e-11 relative with the same cycle counts (the drop-in bar
against the reference stays 1e-10), mixed within 1e-6; and it must take
launches away."""
import numpy as np
import pytest

from helpers import rel_err
from nabla_b200 import abi, cases, solver
from test_gpu_vtail import _channel_run, _with_tuning

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_channel_grid_vcycle_matches_per_sweep(ctx, precision):
    ref, it_ref, n_ref = _with_tuning(ctx, dict(vgrid=0), lambda: _channel_run(ctx, precision))
    got, it_got, n_got = _with_tuning(ctx, dict(vgrid=1), lambda: _channel_run(ctx, precision))
    tol = 1e-11 if precision == abi.PRECISION_FP64 else 1e-6
    for a in range(4):
        assert rel_err(got[a], ref[a]) < tol, (a, rel_err(got[a], ref[a]))
    if precision == abi.PRECISION_FP64:
        assert it_got == it_ref
    else:
        assert all(abs(x - y) <= 1 for x, y in zip(it_got, it_ref))
    assert n_got < n_ref


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_periodic_tgv_grid_vcycle_matches_per_sweep(ctx, precision):
    """Singular system: pending means after every sweep, coarsest Jacobi-CG."""
    g, cfg = cases.taylor_green(32)

    def run():
        ns = solver.NSSolver(g, cfg, precision=precision, ctx=ctx)
        ns.set_state(*cases.taylor_green_state(g))
        its = [ns.step(0.07).poisson_iters for _ in range(3)]
        st = ns.get_state()
        ns.close()
        return st, its

    ref, it_ref = _with_tuning(ctx, dict(vgrid=0), run)
    got, it_got = _with_tuning(ctx, dict(vgrid=1), run)
    tol = 1e-11 if precision == abi.PRECISION_FP64 else 1e-6
    for a in range(4):
        assert rel_err(got[a], ref[a]) < tol, (a, rel_err(got[a], ref[a]))
    if precision == abi.PRECISION_FP64:
        assert it_got == it_ref


def test_grid_vcycle_poisson_solve_matches_oracle(ctx, orc):
    from helpers import channel_block_grid
    g = channel_block_grid()
    b = np.random.default_rng(12345).uniform(-1, 1, g.ncell)
    xo, ro = orc.poisson(g, b, 1e-10, 200)
    x, rep = _with_tuning(ctx, dict(vgrid=1), lambda: solver.MgPoisson(1e-10, 200, ctx=ctx).solve(g, b))
    assert rep.iterations == ro.iterations and rep.converged
    assert rel_err(x, xo) < 1e-10
