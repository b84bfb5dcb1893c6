"""Cluster-resident V-cycle tail (nb_tuning.tail_bricks): the coarse end of
every V-cycle runs as one thread-block-cluster launch, phase by phase. Each
phase is the launch path's own per-brick code, so on a system without
pending means (an outlet makes it non-singular) the step is bitwise equal to
the per-sweep launches; on singular systems the pending means are summed in
another order (FP64 within 1e-9, mixed within 1e-6 of the per-sweep form).
The tail must also take launches away."""
import numpy as np
import pytest

from amr_helpers import refine_where
from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu


def _with_tuning(ctx, tuning, fn):
    ctx.set_tuning(**tuning)
    try:
        return fn()
    finally:
        ctx.set_tuning(**solver.default_tuning())


def _channel_run(ctx, precision, nsteps=3):
    """Two-level octree channel (inlet / outlet / walls): MG levels of 30, 16
    and 2 bricks above an exact 128-cell coarsest solve."""
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = amr.base_leaves((4, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 0)).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    cfg = cases.flow_config(reynolds=1000.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    ac = amr.AmrCase(mesh, cfg, precision=precision)
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append((1.0 if a == 0 else 0.0) + 0.05 * np.sin(6 * x + 2 * a) * np.cos(5 * y) * np.cos(4 * z))
    st.append(np.zeros(ac.sizes[3]))
    ac.set_state(*st)
    n0 = ctx.launches
    iters = []
    for _ in range(nsteps):
        rep = ac.step(0.004)
        assert rep.converged and rep.divergence_max <= 1e-8
        iters.append(rep.poisson_iters)
    return ac.get_state(), iters, ctx.launches - n0


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("tail", [2, 16])
def test_channel_tail_is_bitwise_equal(ctx, precision, tail):
    ref, it_ref, n_ref = _with_tuning(ctx, dict(vgrid=0, tail_bricks=0), lambda: _channel_run(ctx, precision))
    got, it_got, n_got = _with_tuning(ctx, dict(vgrid=0, tail_bricks=tail), lambda: _channel_run(ctx, precision))
    assert it_got == it_ref
    for a in range(4):
        assert np.array_equal(got[a], ref[a])
    assert n_got < n_ref


@pytest.mark.parametrize("precision,tol", [(abi.PRECISION_FP64, 1e-9), (abi.PRECISION_MIXED, 1e-6)])
def test_singular_uniform_box_with_cg_coarsest(ctx, precision, tol):
    """Periodic TGV 32^3 (singular: pending means on every level): MG levels of
    64 and 8 bricks above the one-CTA CG solve of the 8^3 coarsest level."""
    def run():
        g, cfg = cases.taylor_green(32)
        ns = solver.NSSolver(g, cfg, precision=precision, ctx=ctx)
        ns.set_state(*cases.taylor_green_state(g))
        for _ in range(2):
            rep = ns.step(0.05)
            assert rep.converged
        return ns.u_face(), ns.pressure()
    u0, p0 = _with_tuning(ctx, dict(vgrid=0, tail_bricks=0), run)
    u1, p1 = _with_tuning(ctx, dict(vgrid=0, tail_bricks=8), run)
    assert np.abs(u1 - u0).max() <= tol * np.abs(u0).max()
    assert np.abs(p1 - p0).max() <= tol * np.abs(p0).max()


@pytest.mark.parametrize("precision,tol", [(abi.PRECISION_FP64, 1e-9), (abi.PRECISION_MIXED, 1e-6)])
def test_singular_three_level_box_whole_hierarchy_in_the_tail(ctx, precision, tol):
    """Closed lid box, 3 octree levels with solids (singular, composite levels
    with coarse-fine couplings, exact coarsest solve): with tail_bricks large
    every level below the finest is in the tail."""
    geom = amr.make_geom((2, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2,
                         [dict(type=abi.BC_WALL) for _ in range(3)] +
                         [dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))] +
                         [dict(type=abi.BC_WALL) for _ in range(2)])
    lv = amr.base_leaves((2, 2, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 0 and z == 0)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 1 and z == 1)
    solid = (np.random.default_rng(3).random(lv.shape[0] * 512) < 0.04).astype(np.uint8)
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_WENO5, poisson_tol=1e-10)

    def run():
        mesh = amr.AmrMesh(geom, lv, solid=solid, ctx=ctx)
        ac = amr.AmrCase(mesh, cfg, precision=precision)
        rng = np.random.default_rng(11)
        ac.set_state(*[0.1 * rng.standard_normal(n) for n in ac.sizes[:3]], np.zeros(ac.sizes[3]))
        for _ in range(2):
            rep = ac.step(0.004)
            assert rep.converged and rep.divergence_max <= 1e-8
        return ac.get_state()
    ref = _with_tuning(ctx, dict(vgrid=0, tail_bricks=0), run)
    got = _with_tuning(ctx, dict(vgrid=0, tail_bricks=4096), run)
    scale = max(np.abs(ref[a]).max() for a in range(3))
    for a in range(3):
        assert np.abs(got[a] - ref[a]).max() <= tol * scale


def test_cases_with_different_tail_sizes_coexist(ctx):
    """The tail kernel's shared-memory limit is shared by every solver: a case
    whose tail needs more shared memory must still step after a case with a
    smaller tail was built."""
    g, cfg = cases.taylor_green(32)
    big = solver.NSSolver(g, cfg, ctx=ctx)  # tail: 8 + 1 bricks and the CG scratch
    big.set_state(*cases.taylor_green_state(g))
    assert big.step(0.05).converged
    _channel_run(ctx, abi.PRECISION_FP64, nsteps=1)  # tail: 2 + 1 bricks, exact solve
    assert big.step(0.05).converged
