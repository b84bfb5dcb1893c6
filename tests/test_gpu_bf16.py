"""BF16 storage of the coarse levels' restricted residuals (nb_tuning.
coarse_bf16, mixed form): the levels between the finest and the cluster tail
keep b in BF16 (rounded to nearest, widened to FP32 on every read); the
arithmetic stays FP32 and the outer PCG FP64, so the solve still meets its
tolerance on the true residual and the step's velocity stays within the mixed
form's bar (1e-6 relative) of the FP32-residual form."""
import numpy as np
import pytest

from helpers import rel_err
from nabla_b200 import abi, cases, solver
from test_gpu_vtail import _channel_run, _with_tuning

pytestmark = pytest.mark.gpu


def test_channel_step_with_bf16_residuals(ctx):
    ref, it_ref, _ = _with_tuning(ctx, dict(coarse_bf16=0), lambda: _channel_run(ctx, abi.PRECISION_MIXED))
    got, it_got, _ = _with_tuning(ctx, dict(coarse_bf16=1), lambda: _channel_run(ctx, abi.PRECISION_MIXED))
    for a in range(3):
        assert rel_err(got[a], ref[a]) < 1e-6
    assert all(abs(x - y) <= 3 for x, y in zip(it_got, it_ref))


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_bf16_poisson_solve_meets_tolerance(ctx, tol):
    g, _ = cases.taylor_green(32)
    b = np.random.default_rng(11).standard_normal(g.ncell)
    b -= b.mean()

    def run(prec, bf16):
        return _with_tuning(ctx, dict(coarse_bf16=bf16, tail_bricks=0),
                            lambda: solver.MgPoisson(tol, 300, precision=prec, ctx=ctx).solve(g, b))

    x, rep = run(abi.PRECISION_MIXED, 1)
    assert rep.converged and rep.residual <= tol
    xd, _ = run(abi.PRECISION_FP64, 0)
    assert rel_err(x, xd) < max(1e-6, 1e4 * tol)
