"""GPU parity of the full SSP-RK3 / WENO-5 / MG-PCG step (NSSolver seam)
through the C ABI against the golden fixtures and the oracle restatement.

Tolerance: 1e-10 relative (max-norm) in u, v, w and p, the drop-in bar for
the plain FP64 form; Poisson cycle counts must match exactly.
"""
import os

import numpy as np
import pytest

from helpers import mixed_bc_grid, rel_err
from nabla_b200 import abi, cases, solver

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_small.npz"))
TOL = 1e-10


def test_tgv16_matches_reference_golden(ctx):
    g, cfg = cases.taylor_green(16)
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    ns.set_state(*cases.taylor_green_state(g))
    dt = ns.compute_dt()
    assert dt == pytest.approx(float(GOLD["tgv16_dt"]), rel=1e-14)
    for s in (1, 2):
        r = ns.step(dt)
        assert r.poisson_iters == int(GOLD[f"tgv16_s{s}_rep"][0])
        for f, a in zip("uvwp", ns.get_state()):
            assert rel_err(a, GOLD[f"tgv16_s{s}_{f}"]) < TOL, (s, f)
        assert r.continuity_residual == pytest.approx(GOLD[f"tgv16_s{s}_rep"][1], rel=1e-3, abs=1e-15)


def test_cube_matches_reference_golden(ctx):
    """Wall-mounted cube (inlet, outlet, walls, periodic span, solid), CFL dt."""
    g, cfg = cases.wall_mounted_cube(2, 200.0)
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    ns.initialize()
    for s in (1, 2):
        r = ns.step()
        dt, iters, cd, cl, mass = GOLD[f"cube2_s{s}_rep"]
        assert r.dt == pytest.approx(dt, rel=1e-13)
        assert r.poisson_iters == int(iters)
        assert r.cd == pytest.approx(cd, rel=1e-8, abs=1e-12)
        for f, a in zip("uvwp", ns.get_state()):
            assert rel_err(a, GOLD[f"cube2_s{s}_{f}"]) < TOL, (s, f)


def _run_pair(ctx, orc, g, cfg, nsteps, init="initialize", dt=0.0):
    a = solver.NSSolver(g, cfg, ctx=ctx)
    b = orc.ns(g, cfg)
    if init == "initialize":
        a.initialize()
        b.initialize()
    else:
        st = init
        a.set_state(*st)
        b.set_state(*st)
    for _ in range(nsteps):
        ra, rb = a.step(dt), b.step(dt)
        assert ra.poisson_iters == rb.poisson_iters
        assert ra.dt == pytest.approx(rb.dt, rel=1e-12)
    for f, x, y in zip("uvwp", a.get_state(), b.get_state()):
        assert rel_err(x, y) < TOL, f
    return ra, rb


def test_tgv32_three_steps(ctx, orc):
    g, cfg = cases.taylor_green(32)
    st = cases.taylor_green_state(g)
    ra, rb = _run_pair(ctx, orc, g, cfg, 3, init=st, dt=0.07)
    assert ra.divergence_max < 1e-8


@pytest.mark.parametrize("kind", ["lid", "channel_weno", "channel_central"])
def test_2d_reference_cases(ctx, orc, kind):
    if kind == "lid":
        g, cfg = cases.lid_cavity(24, 100.0)
        cfg.poisson_tol = 1e-10
    else:
        g, cfg = cases.channel(48, 16, 200.0)
        cfg.convection = abi.CONV_WENO5 if kind == "channel_weno" else abi.CONV_CENTRAL
        cfg.poisson_tol = 1e-9
    _run_pair(ctx, orc, g, cfg, 4)


def test_mixed_bc_partial_bricks(ctx, orc):
    g = mixed_bc_grid()
    cfg = cases.flow_config(reynolds=50.0, convection=abi.CONV_WENO5, poisson_tol=1e-10)
    _run_pair(ctx, orc, g, cfg, 3)


def test_lid_cavity_projection_continuity(ctx):
    """core/tests/test_flow.cpp:161-172: continuity residual < 1e-7 after 5 steps."""
    g, cfg = cases.lid_cavity(24, 100.0)
    cfg.poisson_tol = 1e-10
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    ns.initialize()
    for _ in range(5):
        r = ns.step()
    assert r.continuity_residual < 1e-7


def test_restart_is_bit_exact(ctx):
    """core/tests/test_flow.cpp:214-247 on the device: 8 steps straight equal
    4 steps + state download/upload + 4 steps, bit for bit."""
    g, cfg = cases.channel(32, 16, 100.0)
    cfg.poisson_tol = 1e-9
    a = solver.NSSolver(g, cfg, ctx=ctx)
    a.initialize()
    for _ in range(8):
        a.step()
    gold = a.get_state()
    b = solver.NSSolver(g, cfg, ctx=ctx)
    b.initialize()
    for _ in range(4):
        b.step()
    st = b.get_state()
    step, t, dtl = b.clock()
    c = solver.NSSolver(g, cfg, ctx=ctx)
    c.initialize()
    c.set_state(*st, step=step, t=t, dt_last=dtl)
    for _ in range(4):
        c.step()
    for x, y in zip(c.get_state(), gold):
        assert np.array_equal(x, y)


def test_state_roundtrip_and_errors(ctx):
    g, cfg = cases.taylor_green(16)
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    st = cases.random_state(g, 5)
    ns.set_state(*st, step=3, t=0.5, dt_last=0.1)
    for x, y in zip(ns.get_state(), st):
        assert np.array_equal(x, y)
    assert ns.clock() == (3, 0.5, 0.1)
    # read-back into caller buffers (the end-to-end path uses pinned ones)
    outs = [np.full(x.size, np.nan) for x in st]
    got = ns.get_state(outs)
    for x, o, y in zip(got, outs, st):
        assert x is o and np.array_equal(o, y)
    with pytest.raises(solver.NablaError):
        ns.get_state([o[:-1] for o in outs])
    with pytest.raises(solver.NablaError):
        ns.get_state([o.astype(np.float32) for o in outs])
    with pytest.raises(solver.NablaError):
        ns.set_state(st[0][:-1], *st[1:])
    bad = cases.Grid(0, 4, 4, 1.0, 1.0, 1.0)
    with pytest.raises(solver.NablaError) as e:
        solver.NSSolver(bad, cfg, ctx=ctx)
    assert e.value.status == abi.NB_ERR_BAD_ARG


def test_launch_counter_counts_cuda_kernels(ctx):
    g, cfg = cases.taylor_green(16)
    ns = solver.NSSolver(g, cfg, ctx=ctx)
    ns.set_state(*cases.taylor_green_state(g))
    before = ctx.launches
    ns.step(0.05)
    assert ctx.launches - before > 50


def test_graph_and_direct_launch_paths_agree_bitwise(ctx):
    """The step runs as one CUDA graph (device-side MG-PCG loop); with kernel
    profiling on it runs as direct launches. Both must give identical bits."""
    import ctypes as C
    g, cfg = cases.wall_mounted_cube(2, 200.0)
    a = solver.NSSolver(g, cfg, ctx=ctx)
    b = solver.NSSolver(g, cfg, ctx=ctx)
    a.initialize()
    b.initialize()
    for _ in range(3):
        ra = a.step()
    ctx.lib.nb_ctx_profile(ctx.h, b"vgrid" if ctx.tuning["vgrid"] else b"smooth")
    try:
        for _ in range(3):
            rb = b.step()
    finally:
        ms, nl, nb = C.c_double(), C.c_uint64(), C.c_double()
        ctx.lib.nb_ctx_profile_read(ctx.h, C.byref(ms), C.byref(nl), C.byref(nb))
        ctx.lib.nb_ctx_profile(ctx.h, None)
    assert nl.value > 0 and ms.value > 0
    assert ra.poisson_iters == rb.poisson_iters
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
