"""GPU parity of the multi-level octree MAC step against the oracle's
restatement (oracle/restate_amr.c, pinned to the uniform restatement in
test_oracle_amr.py).

Both run the same steps with a fixed dt from the same state; the GPU solves
the pressure by MG-PCG to 1e-12, the oracle by Jacobi-CG to 1e-13, so the
comparison tolerance is 1e-9 relative (max norm) on every stored face
velocity and on the pressure.
"""
import numpy as np
import pytest

from amr_helpers import refine_where
from helpers import rel_err
from nabla_b200 import abi, amr, cases

pytestmark = pytest.mark.gpu
TOL = 1e-9


def run_pair(ctx, orc, geom, leaves, cfg, solid, field, nsteps, dt):
    mesh = amr.AmrMesh(geom, leaves, solid=solid, ctx=ctx)
    ac = amr.AmrCase(mesh, cfg)
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append(field(a, x, y, z))
    st.append(np.zeros(ac.sizes[3]))
    ac.set_state(*st)
    A = orc.amr(geom, leaves, cfg, solid=solid)
    idx = [ac.face_index(a) for a in range(3)]
    cidx = amr.cell_coords(mesh.leaves)
    # the oracle takes its leaves and solids in the input order; set by position
    for a in range(3):
        A.set(a, idx[a], st[a])
    for _ in range(nsteps):
        r = ac.step(dt)
        A.step(dt, 1e-13)
        assert r.converged
    got = ac.get_state()
    for a in range(3):
        assert rel_err(got[a], A.get(a, idx[a])) < TOL, ("uvw"[a], rel_err(got[a], A.get(a, idx[a])))
    assert rel_err(got[3], A.get(3, cidx)) < TOL


def _field(mean=(1.0, 0.0, 0.0), amp=0.1):
    def f(a, x, y, z):
        return mean[a] + amp * np.sin(5 * x + 1.3 * a) * np.cos(4 * y + 0.5) * np.cos(3 * z + 0.2 * a)
    return f


def test_two_level_channel_with_solids_matches_oracle(ctx, orc):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = refine_where(geom, amr.base_leaves((4, 2, 2)), lambda L, x, y, z: y == 1 and z == 0)
    lev, i, j, k = amr.cell_coords(lv)
    h = 1.0 / 16 / (2.0 ** lev)
    cx, cy, cz = (i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h
    solid = ((np.abs(cx - 1.0) < 0.1) & (np.abs(cy - 0.55) < 0.12) & (cz < 0.3)).astype(np.uint8)
    cfg = cases.flow_config(reynolds=500.0, convection=abi.CONV_WENO5, poisson_tol=1e-12, poisson_max_iters=400)
    run_pair(ctx, orc, geom, lv, cfg, solid, _field(), 2, 0.01)


def test_three_level_periodic_box_matches_oracle(ctx, orc):
    geom = amr.make_geom((2, 2, 2), (0.25, 0.25, 0.25), 2, cases.periodic_faces())
    lv = amr.base_leaves((2, 2, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 1)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 2 and z == 1)
    cfg = cases.flow_config(reynolds=300.0, convection=abi.CONV_WENO5, poisson_tol=1e-12, poisson_max_iters=400)
    run_pair(ctx, orc, geom, lv, cfg, None, _field((0.3, -0.2, 0.1), 0.3), 2, 0.02)


def test_three_level_lid_box_with_solids_matches_oracle(ctx, orc):
    geom = amr.make_geom((2, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2,
                         [dict(type=abi.BC_WALL) for _ in range(3)] +
                         [dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))] +
                         [dict(type=abi.BC_WALL) for _ in range(2)])
    lv = amr.base_leaves((2, 2, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 0 and z == 0)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 1 and z == 1)
    solid = (np.random.default_rng(3).random(lv.shape[0] * 512) < 0.04).astype(np.uint8)
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_CENTRAL, poisson_tol=1e-12, poisson_max_iters=400)
    run_pair(ctx, orc, geom, lv, cfg, solid, _field((0.0, 0.0, 0.0), 0.2), 2, 0.004)


def test_three_level_channel_refined_at_inlet_and_outlet_matches_oracle(ctx, orc):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_PARABOLIC, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2, faces)
    lv = refine_where(geom, amr.base_leaves((4, 2, 2)), lambda L, x, y, z: x in (0, 3))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x in (0, 7) and y == 1)
    cfg = cases.flow_config(reynolds=400.0, convection=abi.CONV_WENO5, poisson_tol=1e-12, poisson_max_iters=400)
    run_pair(ctx, orc, geom, lv, cfg, None, _field(), 2, 0.004)
