"""Batched stepping (nb_batch_step): each step of a set of independent cases
is one CUDA graph launch whose branches are the cases' own steps. A case's
result must not depend on its company: stepping it in a batch must give the
same bits as stepping it alone (the same kernels run, only concurrently)."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu


def _tgv(ctx, n=16, precision=abi.PRECISION_FP64):
    g, cfg = cases.taylor_green(n)
    ns = solver.NSSolver(g, cfg, precision=precision, ctx=ctx)
    ns.set_state(*cases.taylor_green_state(g))
    return ns


def _channel(ctx, precision=abi.PRECISION_FP64, seed=0):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    geom = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 1, faces)
    lv = amr.base_leaves((4, 2, 2))
    lv = amr.refine(geom, lv, ((lv[:, 1] == 1 + seed % 2) & (lv[:, 2] == 0)).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    cfg = cases.flow_config(reynolds=1000.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    ac = amr.AmrCase(mesh, cfg, precision=precision)
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append((1.0 if a == 0 else 0.0) + 0.05 * np.sin(6 * x + 2 * a + seed) * np.cos(5 * y) * np.cos(4 * z))
    st.append(np.zeros(ac.sizes[3]))
    ac.set_state(*st)
    ac._mesh_keepalive = mesh
    return ac


def _mix(ctx):
    return [_tgv(ctx), _channel(ctx, seed=0), _channel(ctx, abi.PRECISION_MIXED, seed=1), _tgv(ctx, 24)]


def test_batch_gives_the_same_bits_as_single_steps(ctx):
    a, b = _mix(ctx), _mix(ctx)
    ra = solver.batch_step(a, 0.0, 3)
    for c in b:
        for _ in range(3):
            rb = c.step()
    for x, y, r in zip(a, b, ra):
        for s, t in zip(x.get_state(), y.get_state()):
            assert np.array_equal(s, t)
    assert ra[-1].poisson_iters == rb.poisson_iters
    assert all(r.converged for r in ra)


def test_batch_alternates_with_single_steps_and_survives_case_removal(ctx):
    a, b = _mix(ctx), _mix(ctx)
    solver.batch_step(a, 0.0, 1)
    a[1].step()  # parities now differ between cases
    solver.batch_step(a, 0.0, 2)
    for i, c in enumerate(b):
        for _ in range(3 + (i == 1)):
            c.step()
    for x, y in zip(a, b):
        for s, t in zip(x.get_state(), y.get_state()):
            assert np.array_equal(s, t)
    gone = a.pop(2)
    gone.close()
    reps = solver.batch_step(a, 0.0, 1)
    assert len(reps) == 3 and all(r.converged for r in reps)


def test_batch_fixed_dt_and_bad_arguments(ctx):
    a = [_tgv(ctx), _tgv(ctx)]
    reps = solver.batch_step(a, 0.05, 2)
    assert all(r.dt == pytest.approx(0.05) for r in reps)
    with pytest.raises(solver.NablaError):
        solver.batch_step([a[0], a[0]], 0.0, 1)


def test_context_destroyed_before_its_cases():
    """Cases and meshes hold their context: destroying the context handle first
    (as a garbage collector may at interpreter exit) leaves them usable to
    destroy, and the batch graphs that name them are released with them."""
    own = solver.Context(0)
    a, b = _channel(own, seed=0), _channel(own, seed=1)
    solver.batch_step([a, b], nsteps=1)
    mesh = a._mesh_keepalive
    own.close()
    a.close()
    mesh.close()
    b.close()
    b._mesh_keepalive.close()
