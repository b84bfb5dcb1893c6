"""GPU parity: the -Laplacian and the MG-PCG pressure solve (the PoissonSolver
seam) through the C ABI, against the oracle restatement and the golden
fixtures from the reference.

Tolerances: the operator is exact up to FMA rounding (1e-13 relative); a
solve matches the FP64 oracle to 1e-10 relative with the same cycle count
(the plain form restates the reference algorithm, so the iterates agree to
rounding); the mixed form must reach the requested tolerance.
"""
import os

import numpy as np
import pytest

from helpers import channel_block_grid, closed_box_grid, mixed_bc_grid, periodic2d_grid, rel_err
from nabla_b200 import abi, cases, solver

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_small.npz"))


def test_apply_a_golden_partial_bricks(ctx):
    g = mixed_bc_grid()
    got = solver.apply_a(g, GOLD["applyA_mixed_x"], ctx)
    assert rel_err(got, GOLD["applyA_mixed_Ax"]) < 1e-13


@pytest.mark.parametrize("make", [lambda: cases.taylor_green(32)[0], channel_block_grid,
                                  lambda: periodic2d_grid(24), closed_box_grid,
                                  lambda: mixed_bc_grid(19, 7, 17, seed=9)])
def test_apply_a_matches_oracle(ctx, orc, make):
    g = make()
    x = np.random.default_rng(4).uniform(-1, 1, g.ncell)
    assert rel_err(solver.apply_a(g, x, ctx), orc.apply_a(g, x)) < 1e-13


def test_mg_reference_channel_block(ctx):
    """core/tests/test_flow.cpp:63-117 on the GPU: converged, residual < 1e-8,
    <= 50 cycles, RMS error < 1e-6; same cycles and solution as the reference."""
    g = channel_block_grid()
    x, rep = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(g, GOLD["mg_channel_b"])
    it, res, conv = GOLD["mg_channel_rep"]
    assert rep.converged and rep.residual < 1e-8 and rep.iterations <= 50
    assert rep.iterations == int(it)
    assert np.sqrt(np.mean((x - GOLD["mg_channel_xexact"]) ** 2)) < 1e-6
    assert rel_err(x, GOLD["mg_channel_x"]) < 1e-10


def test_mg_reference_periodic_singular(ctx):
    """core/tests/test_flow.cpp:119-159 (singular periodic 24x24)."""
    g = periodic2d_grid(24)
    x, rep = solver.MgPoisson(1e-12, 100, ctx=ctx).solve(g, GOLD["mg_periodic_b"])
    assert rep.residual < 1e-8 and rep.iterations <= 50
    assert rep.iterations == int(GOLD["mg_periodic_rep"][0])
    assert rel_err(x, GOLD["mg_periodic_x"]) < 1e-9


def test_mg_closed_box_with_solids(ctx):
    g = closed_box_grid()
    x, rep = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(g, GOLD["mg_box_b"])
    assert rep.iterations == int(GOLD["mg_box_rep"][0])
    assert rel_err(x, GOLD["mg_box_x"]) < 1e-10


@pytest.mark.parametrize("make,tol", [(lambda: cases.taylor_green(32)[0], 1e-10),
                                      (lambda: mixed_bc_grid(19, 7, 17, seed=9), 1e-10),
                                      (lambda: cases.wall_mounted_cube(2, 100.0)[0], 1e-12)])
def test_mg_matches_oracle(ctx, orc, make, tol):
    g = make()
    b = np.random.default_rng(8).standard_normal(g.ncell) * (1 - g.solid)
    xo, ro = orc.poisson(g, b, tol, 200)
    x, rep = solver.MgPoisson(tol, 200, ctx=ctx).solve(g, b)
    assert rep.iterations == ro.iterations
    assert rep.converged == bool(ro.converged)
    assert rel_err(x, xo) < 1e-9


def test_mg_zero_rhs_early_exit(ctx):
    g = channel_block_grid()
    x, rep = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(g, np.zeros(g.ncell))
    assert rep.iterations == 0 and rep.converged and np.all(x == 0)


def test_mg_max_cycles_reported_not_raised(ctx, orc):
    g = cases.taylor_green(32)[0]
    b = np.random.default_rng(1).standard_normal(g.ncell)
    x, rep = solver.MgPoisson(1e-14, 2, ctx=ctx).solve(g, b)
    xo, ro = orc.poisson(g, b, 1e-14, 2)
    assert rep.iterations == 2 and not rep.converged
    assert rel_err(x, xo) < 1e-9


def test_mg_mixed_precision_reaches_tolerance(ctx, orc):
    g = cases.taylor_green(32)[0]
    b = np.random.default_rng(2).standard_normal(g.ncell)
    xo, ro = orc.poisson(g, b, 1e-10, 200)
    x, rep = solver.MgPoisson(1e-10, 200, precision=abi.PRECISION_MIXED, ctx=ctx).solve(g, b)
    assert rep.converged and rep.residual <= 1e-10
    assert rep.iterations <= ro.iterations + 3
    assert rel_err(x, xo) < 1e-8


def test_mg_deterministic(ctx):
    g = channel_block_grid()
    b = GOLD["mg_channel_b"]
    x1, _ = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(g, b)
    x2, _ = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(g, b)
    assert np.array_equal(x1, x2)
