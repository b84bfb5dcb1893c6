"""Checkpoints on the GPU (nb_case_write_checkpoint / nb_case_read_checkpoint):
restart is bit-exact (core/tests/test_flow.cpp:214-247 restated: 8 steps
against 4 + checkpoint + fresh solver + 4), NBFCK01 files move between the
compiled reference and this library in both directions, and octree cases
restart bit for bit from NBFAMR1 files of their own mesh only."""
import ctypes as C

import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu


def _channel_grid():
    grid, cfg = cases.channel(32, 16, 100.0, 1.0)
    cfg.poisson_tol = 1e-9
    return grid, cfg


def _state(ns):
    return [np.array(a) for a in ns.get_state()]


def test_uniform_restart_is_bit_exact(ctx, tmp_path):
    grid, cfg = _channel_grid()
    gold = solver.NSSolver(grid, cfg, ctx=ctx)
    gold.initialize()
    for _ in range(8):
        gold.step()
    a = solver.NSSolver(grid, cfg, ctx=ctx)
    a.initialize()
    for _ in range(4):
        a.step()
    path = tmp_path / "restart.ckpt"
    a.write_checkpoint(path)
    assert solver.checkpoint_info(path)["step"] == 4
    b = solver.NSSolver(grid, cfg, ctx=ctx)
    b.initialize()
    b.read_checkpoint(path)
    for _ in range(4):
        rep = b.step()
    assert rep.step == 8
    for x, y in zip(_state(b), _state(gold)):
        assert np.array_equal(x, y)


def test_checkpoints_move_between_reference_and_gpu(ctx, ref, tmp_path):
    grid, cfg = _channel_grid()
    r = ref.ns(grid, cfg)
    r.initialize()
    for _ in range(3):
        r.step()
    path = tmp_path / "from_ref.ckpt"
    r.write_checkpoint(path)
    g = solver.NSSolver(grid, cfg, ctx=ctx)
    g.read_checkpoint(path)
    for x, y in zip(_state(g), r.get_state()):
        assert np.array_equal(x, y)  # the file carries every bit
    for _ in range(2):
        g.step()
        r.step()
    for x, y in zip(_state(g), r.get_state()):
        assert np.abs(x - y).max() <= 1e-10 * max(np.abs(y).max(), 1e-30)
    back = tmp_path / "from_gpu.ckpt"
    g.write_checkpoint(back)
    r2 = ref.ns(grid, cfg)
    r2.initialize()
    r2.read_checkpoint(back)
    for x, y in zip(r2.get_state(), _state(g)):
        assert np.array_equal(x, y)


def _amr_channel(ctx, refine_col):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = amr.base_leaves((4, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == refine_col) & (lv[:, 2] == 0)).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    cfg = cases.flow_config(reynolds=1000.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    return mesh, cfg


def _amr_case(mesh, cfg, precision):
    ac = amr.AmrCase(mesh, cfg, precision=precision)
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append((1.0 if a == 0 else 0.0) + 0.05 * np.sin(6 * x + 2 * a) * np.cos(5 * y) * np.cos(4 * z))
    st.append(np.zeros(ac.sizes[3]))
    ac.set_state(*st)
    return ac


def _clock(ctx, case):
    step, t, dt = C.c_int(), C.c_double(), C.c_double()
    ctx.lib.nb_case_get_clock(case.h, C.byref(step), C.byref(t), C.byref(dt))
    return step.value, t.value, dt.value


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_octree_restart_is_bit_exact(ctx, tmp_path, precision):
    """Bit for bit when the initial guesses are functions of the state: the FP64
    form (zero start) and the mixed form with the scaled-pressure start."""
    ctx.set_tuning(warm_start=1)
    try:
        _octree_restart(ctx, tmp_path, precision, exact=True)
    finally:
        ctx.set_tuning(**solver.default_tuning())


def test_octree_restart_with_history_start_agrees(ctx, tmp_path):
    """The mixed form's default history start is not part of the checkpoint: the
    restarted run agrees with the continuous one to the solver tolerance."""
    _octree_restart(ctx, tmp_path, abi.PRECISION_MIXED, exact=False)


def _octree_restart(ctx, tmp_path, precision, exact):
    mesh, cfg = _amr_channel(ctx, 1)
    gold = _amr_case(mesh, cfg, precision)
    for _ in range(6):
        gold.step()
    a = _amr_case(mesh, cfg, precision)
    for _ in range(3):
        a.step()
    path = tmp_path / "octree.ckpt"
    a.write_checkpoint(path)
    info = solver.checkpoint_info(path)
    assert info["kind"] == "octree" and info["leaves"] == mesh.leaves.shape[0] and info["step"] == 3
    b = amr.AmrCase(mesh, cfg, precision=precision)
    b.read_checkpoint(path)
    assert _clock(ctx, b) == _clock(ctx, a)
    for _ in range(3):
        b.step()
    if exact:
        assert _clock(ctx, b) == _clock(ctx, gold)
    else:
        assert _clock(ctx, b)[0] == _clock(ctx, gold)[0]
    for x, y in zip(b.get_state(), gold.get_state()):
        if exact:
            assert np.array_equal(x, y)
        else:
            assert np.abs(x - y).max() <= 1e-6 * max(np.abs(y).max(), 1.0)


def test_octree_checkpoint_checks_the_mesh(ctx, tmp_path):
    mesh_a, cfg = _amr_channel(ctx, 1)
    mesh_b, _ = _amr_channel(ctx, 2)
    a = _amr_case(mesh_a, cfg, abi.PRECISION_FP64)
    path = tmp_path / "a.ckpt"
    a.write_checkpoint(path)
    b = _amr_case(mesh_b, cfg, abi.PRECISION_FP64)
    with pytest.raises(solver.NablaError, match="leaf list differs"):
        b.read_checkpoint(path)
    grid, ucfg = _channel_grid()
    u = solver.NSSolver(grid, ucfg, ctx=ctx)
    u.initialize()
    upath = tmp_path / "u.ckpt"
    u.write_checkpoint(upath)
    with pytest.raises(solver.NablaError, match="not an octree checkpoint"):
        a.read_checkpoint(upath)
    with pytest.raises(solver.NablaError, match="not a uniform-grid checkpoint"):
        u.read_checkpoint(path)
