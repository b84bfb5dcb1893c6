"""GPU tests of the MAC step on octree-AMR meshes (nb_amr_case_*).

* On single-level meshes the AMR step must reproduce the uniform step, which
  is pinned to the reference NSSolver, to 1e-10 relative in every stored face
  velocity and the pressure, with identical Poisson cycle counts and dt.
* On multi-level meshes the projection must leave the discrete divergence at
  the solver tolerance, closed boxes must conserve mass exactly, the graph
  and direct-launch paths must agree bitwise, and the mixed form must track
  the FP64 form.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_err
from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu
TOL = 1e-10


def lex_maps(case: amr.AmrCase, g: cases.Grid):
    """Storage slot -> reference lexicographic index (single-level meshes)."""
    nx, ny = g.nx, g.ny
    maps = []
    for a in range(3):
        lev, i, j, k = case.face_index(a)
        ex, ey = nx + (a == 0), ny + (a == 1)
        maps.append(i + ex * (j + ey * k))
    lev, i, j, k = amr.cell_coords(case.mesh.leaves)
    maps.append(i + nx * (j + ny * k))
    return maps


def single_level_pair(ctx, g, cfg, nb0, state, nsteps, dt=0.0):
    geom = amr.make_geom(nb0, (g.dx, g.dy, g.dz), 0, g.faces, origin=g.origin)
    base = amr.base_leaves(nb0)
    lev, i, j, k = amr.cell_coords(base)
    solid = g.solid[i + g.nx * (j + g.ny * k)]  # 512 bytes per leaf, input order
    mesh = amr.AmrMesh(geom, base, solid=solid, ctx=ctx)
    ac = amr.AmrCase(mesh, cfg)
    maps = lex_maps(ac, g)
    uni = solver.NSSolver(g, cfg, ctx=ctx)
    uni.set_state(*state)
    ac.set_state(*[np.asarray(s)[m] for s, m in zip(state, maps)])
    for _ in range(nsteps):
        ru, ra = uni.step(dt), ac.step(dt)
        assert ra.poisson_iters == ru.poisson_iters
        assert ra.dt == pytest.approx(ru.dt, rel=1e-13)
        assert ra.converged
    su, sa = uni.get_state(), ac.get_state()
    for f, x, y, m in zip("uvwp", sa, su, maps):
        assert rel_err(x, np.asarray(y)[m]) < TOL, (f, rel_err(x, np.asarray(y)[m]))
    return ru, ra


def test_single_level_periodic_tgv_matches_uniform(ctx):
    g, cfg = cases.taylor_green(32)
    single_level_pair(ctx, g, cfg, (4, 4, 4), cases.taylor_green_state(g), 2, dt=0.07)


def _channel_block_grid():
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_PARABOLIC, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL, wall_velocity=(0.3, 0, 0)),
             dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = cases.Grid(32, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    s = g.solid.reshape(16, 16, 32)
    s[6:10, 0:6, 12:18] = 1
    return g


def test_single_level_channel_with_block_matches_uniform(ctx):
    g = _channel_block_grid()
    cfg = cases.flow_config(reynolds=200.0, convection=abi.CONV_WENO5, poisson_tol=1e-10)
    rng = np.random.default_rng(4)
    st = (rng.uniform(0.5, 1.0, 33 * 16 * 16), rng.uniform(-0.1, 0.1, 32 * 17 * 16),
          rng.uniform(-0.1, 0.1, 32 * 16 * 17), np.zeros(32 * 16 * 16))
    w = st[2].reshape(17, 16, 32)
    w[16] = w[0]  # periodic z: the mesh stores one face where the reference keeps two equal copies
    single_level_pair(ctx, g, cfg, (4, 2, 2), st, 2)


def test_single_level_closed_box_central_matches_uniform(ctx):
    faces = [dict(type=abi.BC_WALL) for _ in range(6)]
    faces[3] = dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))  # lid
    g = cases.Grid(16, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    g.solid[np.random.default_rng(2).random(g.ncell) < 0.03] = 1
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_CENTRAL, poisson_tol=1e-10)
    st = cases.random_state(g, 3, amp=0.2)
    single_level_pair(ctx, g, cfg, (2, 2, 2), st, 2)


def _smooth_state(ac, mean_u=1.0):
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append((mean_u if a == 0 else 0.0) + 0.05 * np.sin(6 * x + 2 * a) * np.cos(5 * y) * np.cos(4 * z))
    st.append(np.zeros(ac.sizes[3]))
    return st


def channel_two_level(ctx, precision=abi.PRECISION_FP64):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = amr.base_leaves((4, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 0)).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    cfg = cases.flow_config(reynolds=1000.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    ac = amr.AmrCase(mesh, cfg, precision=precision)
    ac.set_state(*_smooth_state(ac))
    return ac


def test_two_level_channel_projects_to_tolerance(ctx):
    ac = channel_two_level(ctx)
    assert ac.mesh.leaves[:, 0].max() == 1
    for _ in range(3):
        r = ac.step()
        assert r.converged
        assert np.isfinite(r.momentum_residual)
        assert r.divergence_max < 1e-8
        assert r.mass_error < 1e-8


def test_three_level_periodic_box_divergence_free_and_deterministic(ctx):
    geom = amr.make_geom((4, 4, 4), (0.25, 0.25, 0.25), 2, cases.periodic_faces())
    lv = amr.base_leaves((4, 4, 4))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 2)).astype(np.uint8))
    lv = amr.refine(geom, lv, ((lv[:, 0] == 1) & (lv[:, 1] == 3) & (lv[:, 2] == 4) & (lv[:, 3] == 2)).astype(np.uint8))
    assert lv[:, 0].max() == 2
    cfg = cases.flow_config(reynolds=500.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    out = []
    for _ in range(2):
        mesh = amr.AmrMesh(geom, lv, ctx=ctx)
        ac = amr.AmrCase(mesh, cfg)
        ac.set_state(*_smooth_state(ac, mean_u=0.3))
        for _ in range(2):
            r = ac.step()
            assert r.converged and r.divergence_max < 1e-8
        out.append(ac.get_state())
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_closed_box_three_level_conserves_mass(ctx):
    geom = amr.make_geom((2, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2,
                         [dict(type=abi.BC_WALL) for _ in range(5)] +
                         [dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))])
    lv = amr.base_leaves((2, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 0) & (lv[:, 2] == 0) & (lv[:, 3] == 0)).astype(np.uint8))
    lv = amr.refine(geom, lv, ((lv[:, 0] == 1) & (lv[:, 1] == 1) & (lv[:, 2] == 1) & (lv[:, 3] == 1)).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_CENTRAL, poisson_tol=1e-10, cfl=0.5)
    ac = amr.AmrCase(mesh, cfg)
    ac.initialize()
    for _ in range(3):
        r = ac.step()
        assert r.converged and r.divergence_max < 1e-8
        assert r.mass_error == 0.0


def test_amr_graph_and_direct_paths_agree_bitwise(ctx):
    a = channel_two_level(ctx)
    b = channel_two_level(ctx)
    for _ in range(2):
        ra = a.step()
    ctx.lib.nb_ctx_profile(ctx.h, b"rhs_rk")
    try:
        for _ in range(2):
            rb = b.step()
    finally:
        ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
        ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
        ctx.lib.nb_ctx_profile(ctx.h, None)
    assert nl.value == 6
    assert ra.poisson_iters == rb.poisson_iters
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    # read-back into caller buffers gives the same arrays
    outs = [np.full(n, np.nan) for n in b.sizes]
    for x, o in zip(b.get_state(), b.get_state(outs)):
        assert np.array_equal(x, o)
    with pytest.raises(ValueError):
        b.get_state(outs[:3] + [outs[3][:-1]])


def test_two_level_mixed_tracks_fp64(ctx):
    a = channel_two_level(ctx, abi.PRECISION_FP64)
    b = channel_two_level(ctx, abi.PRECISION_MIXED)
    for _ in range(3):
        ra, rb = a.step(), b.step()
    assert rb.converged and rb.divergence_max < 1e-8
    for x, y in zip(b.get_state()[:3], a.get_state()[:3]):
        assert rel_err(x, y) < 1e-5
