"""GPU parity at the configurations' stated sizes, against the CPU oracles.

* Taylor-Green, periodic [0, 2 pi]^3 on the uniform 64^3 MAC grid, FP64,
  nu = 1/1600, WENO-5, fixed dt = computeDt of the initial state (CFL 0.4),
  20 SSP-RK3 steps, MG-PCG to 1e-10: against the reference's own NSSolver
  compiled from its sources (oracle/_ref, core/src/flow/ns_solver.cpp:767-824).
  The same MG-PCG cycle count at every step (the reference's determinism,
  core/tests/test_flow.cpp:214-247, is what makes the comparison exact) and
  u, v, w, p within 1e-10 relative (max norm) after 1, 10 and 20 steps.
* The 3-level obstacle channel mesh itself (workloads.obstacle_channel(0):
  508 leaves, 260,096 cells, 6 seeded boxes, inflow / outlet / walls,
  nu = 1/1000), two steps with a fixed dt (computeDt of the initial state),
  FP64 against the oracle's octree restatement (oracle/restate_amr.c), both
  pressure solves to a relative residual of 1e-13: every stored face velocity
  and the pressure within 1e-10 relative (max norm).
* The mixed form on the same mesh, from the same state, at the channel's own
  solver tolerance (1e-10): its velocity, pressure and post-projection
  divergence errors are stated against the same FP64 oracle result; the bars
  are velocity <= 1e-6 relative and divergence <= 1e-8.
"""
import numpy as np
import pytest

from helpers import rel_err
from nabla_b200 import abi, amr, cases, solver, workloads

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_tgv64_twenty_steps_match_compiled_reference(ctx, ref):
    g, cfg = cases.taylor_green(64)
    st = cases.taylor_green_state(g)
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    ns.set_state(*st)
    rn = ref.ns(g, cfg)
    rn.set_state(*st)
    dt = rn.compute_dt()
    assert ns.compute_dt() == pytest.approx(dt, rel=1e-14)
    for s in range(1, 21):
        a, b = ns.step(dt), rn.step(dt)
        assert a.poisson_iters == b.poisson_iters, (s, a.poisson_iters, b.poisson_iters)
        assert a.converged
        if s in (1, 10, 20):
            for f, x, y in zip("uvwp", ns.get_state(), rn.get_state()):
                assert rel_err(x, y) < TOL, (s, f, rel_err(x, y))
    assert a.divergence_max < 1e-8
    ns.close()


@pytest.fixture(scope="module")
def channel_oracle(orc):
    """The channel mesh, its initial state, dt, and the oracle's state after two steps."""
    w = workloads.obstacle_channel(0)
    ctx = solver.default_context()
    mesh = amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
    probe = amr.AmrCase(mesh, w.config)
    st = w.initial_state(probe)
    probe.set_state(*st)
    dt = probe.compute_dt()
    idx = [probe.face_index(a) for a in range(3)]
    cidx = amr.cell_coords(mesh.leaves)
    probe.close()
    cfg = w.config
    cfg.poisson_tol = 1e-13
    A = orc.amr(w.geom, w.leaves, cfg, solid=w.solid)
    for a in range(3):
        A.set(a, idx[a], st[a])
    divs = [A.step(dt, 1e-13)[0] for _ in range(2)]
    want = [A.get(a, idx[a]) for a in range(3)] + [A.get(3, cidx)]
    yield dict(w=w, mesh=mesh, st=st, dt=dt, want=want, oracle_div=divs)
    mesh.close()


def _run_channel(ctx, c, precision, tol):
    cfg = c["w"].config
    cfg.poisson_tol = tol
    case = amr.AmrCase(c["mesh"], cfg, precision=precision)
    case.set_state(*c["st"])
    reps = [case.step(c["dt"]) for _ in range(2)]
    got = case.get_state()
    case.close()
    return got, reps


def test_channel_mesh_fp64_matches_oracle(ctx, channel_oracle):
    got, reps = _run_channel(ctx, channel_oracle, abi.PRECISION_FP64, 1e-13)
    assert all(r.converged for r in reps)
    for f, x, y in zip("uvwp", got, channel_oracle["want"]):
        assert rel_err(x, y) < TOL, (f, rel_err(x, y))
    assert reps[-1].divergence_max < 1e-8


def test_channel_mesh_mixed_errors_against_oracle(ctx, channel_oracle):
    got, reps = _run_channel(ctx, channel_oracle, abi.PRECISION_MIXED, 1e-10)
    assert all(r.converged for r in reps)
    want = channel_oracle["want"]
    vel = max(rel_err(x, y) for x, y in zip(got[:3], want[:3]))
    pres = rel_err(got[3], want[3])
    print(f"mixed vs FP64 oracle: velocity {vel:.2e}, pressure {pres:.2e}, "
          f"divergence {reps[-1].divergence_max:.2e}")
    assert vel <= 1e-6
    assert reps[-1].divergence_max <= 1e-8
    assert pres <= 1e-4
