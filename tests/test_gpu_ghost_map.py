"""The octree momentum kernel's ghost map (nb_tuning.ghost_map, default 1)
against the ghost walker it records (ghost_map = 0). The map replays, for
every halo point that is not a same-level cell, the affine form the walker
computes there (core/src/flow/ns_solver.cpp:116-219 ghost rules at a level
jump, the periodic wrap, outlet copies, wall reflections); forms with a
constant part (inlet values, moving walls) keep the walker. The two paths
differ only in the order of the form's sum, so the states after several
steps agree to 1e-12 of the velocity scale (FP64), the MG-PCG cycle counts
match, and the case with the map holds more device memory (the map is
built)."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu


def _state(ac, mean_u):
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append((mean_u if a == 0 else 0.0) + 0.05 * np.sin(6 * x + 2 * a) * np.cos(5 * y) * np.cos(4 * z))
    st.append(np.zeros(ac.sizes[3]))
    return st


def _channel():
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = amr.base_leaves((4, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 0)).astype(np.uint8))
    cfg = cases.flow_config(reynolds=1000.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    return geom, lv, cfg, 1.0


def _periodic_three_level():
    geom = amr.make_geom((4, 4, 4), (0.25, 0.25, 0.25), 2, cases.periodic_faces())
    lv = amr.base_leaves((4, 4, 4))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 2)).astype(np.uint8))
    lv = amr.refine(geom, lv, ((lv[:, 0] == 1) & (lv[:, 1] == 3) & (lv[:, 2] == 4) & (lv[:, 3] == 2)).astype(np.uint8))
    cfg = cases.flow_config(reynolds=500.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    return geom, lv, cfg, 0.3


def _lid_box_three_level():
    geom = amr.make_geom((2, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2,
                         [dict(type=abi.BC_WALL) for _ in range(5)] +
                         [dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))])
    lv = amr.base_leaves((2, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 0) & (lv[:, 2] == 0) & (lv[:, 3] == 0)).astype(np.uint8))
    lv = amr.refine(geom, lv, ((lv[:, 0] == 1) & (lv[:, 1] == 1) & (lv[:, 2] == 1) & (lv[:, 3] == 1)).astype(np.uint8))
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.5)
    return geom, lv, cfg, 0.0


def _run(ctx, build, ghost_map, precision, nsteps=3):
    geom, lv, cfg, mean_u = build()
    ctx.set_tuning(ghost_map=ghost_map)
    try:
        mesh = amr.AmrMesh(geom, lv, ctx=ctx)
        ac = amr.AmrCase(mesh, cfg, precision=precision)
        nbytes = int(ctx.lib.nb_case_device_bytes(ac.h))
        ac.set_state(*_state(ac, mean_u))
        cycles = []
        for _ in range(nsteps):
            rep = ac.step()
            assert rep.converged and rep.divergence_max < 1e-8
            cycles.append(rep.poisson_iters)
        out = ac.get_state()
        ac.close()
        mesh.close()
        return out, cycles, nbytes
    finally:
        ctx.set_tuning(**solver.default_tuning())


@pytest.mark.parametrize("build", [_channel, _periodic_three_level, _lid_box_three_level],
                         ids=["channel_inlet_outlet_walls", "periodic_three_levels", "lid_box_three_levels"])
def test_ghost_map_matches_the_walker_fp64(ctx, build):
    walk, c_walk, b_walk = _run(ctx, build, 0, abi.PRECISION_FP64)
    mapd, c_map, b_map = _run(ctx, build, 1, abi.PRECISION_FP64)
    assert b_map > b_walk  # the map is built and held by the case
    assert c_map == c_walk
    scale = max(np.abs(walk[0]).max(), np.abs(walk[1]).max(), np.abs(walk[2]).max())
    for a in range(3):
        assert np.abs(mapd[a] - walk[a]).max() <= 1e-12 * scale, a
    assert np.abs(mapd[3] - walk[3]).max() <= 1e-10 * max(np.abs(walk[3]).max(), 1e-30)


def test_ghost_map_matches_the_walker_mixed(ctx):
    """Mixed form (FP32 tiles): the forms' values round to the same FP32 tile
    values except where an FP64 value lies within an ulp of an FP32 rounding
    boundary, so the states agree to 1e-7 of the velocity scale, ten times
    inside the mixed form's 1e-6 bar."""
    walk, _, _ = _run(ctx, _periodic_three_level, 0, abi.PRECISION_MIXED)
    mapd, _, _ = _run(ctx, _periodic_three_level, 1, abi.PRECISION_MIXED)
    scale = max(np.abs(walk[0]).max(), np.abs(walk[1]).max(), np.abs(walk[2]).max())
    for a in range(3):
        assert np.abs(mapd[a] - walk[a]).max() <= 1e-7 * scale, a
