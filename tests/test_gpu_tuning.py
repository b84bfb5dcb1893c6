"""Tuned launches on the GPU. Every tuning must leave the step converged with
divergence <= 1e-8; FP64 results may move only by reduction order and the
coarse solve (1e-8 relative here), mixed results within 1e-6 of the default.
The autotuner must return a tuning no slower than the default and reuse its
cache."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu


def _channel(ctx, precision):
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
    ac._mesh_keepalive = mesh
    return ac


def _run(ctx, precision, tuning, nsteps=3):
    ctx.set_tuning(**tuning)
    try:
        ac = _channel(ctx, precision)
        for _ in range(nsteps):
            rep = ac.step(0.004)
            assert rep.converged and rep.divergence_max <= 1e-8
        return ac.get_state()[:3]
    finally:
        ctx.set_tuning(**solver.default_tuning())


VARIANTS = [dict(mg_ctas_per_sm=1, rhs_ctas_per_sm=1), dict(halo_mode=1), dict(pdl=0),
            dict(coarse_direct_max=0), dict(coarse_direct_max=512), dict(mg_ctas_per_sm=3, rhs_ctas_per_sm=4),
            dict(threads_per_brick=256, mg_ctas_per_sm=8), dict(threads_per_brick=128, mg_ctas_per_sm=16),
            dict(threads_per_brick=128, mg_ctas_per_sm=5, halo_mode=1)]


@pytest.mark.parametrize("tuning", VARIANTS)
def test_fp64_tuning_keeps_the_solution(ctx, tuning):
    ref = _run(ctx, abi.PRECISION_FP64, {})
    got = _run(ctx, abi.PRECISION_FP64, tuning)
    for a in range(3):
        assert np.abs(got[a] - ref[a]).max() <= 1e-8 * np.abs(ref[0]).max()


@pytest.mark.parametrize("sweeps,smoother", [(1, 0), (3, 0), (1, 1), (2, 1), (3, 1)])
def test_mixed_sweeps_stay_within_tolerance(ctx, sweeps, smoother):
    ref = _run(ctx, abi.PRECISION_FP64, {})
    got = _run(ctx, abi.PRECISION_MIXED, dict(sweeps=sweeps, smoother=smoother))
    for a in range(3):
        assert np.abs(got[a] - ref[a]).max() <= 1e-6 * np.abs(ref[0]).max()


def test_autotune_and_cache(ctx, tmp_path):
    ac = _channel(ctx, abi.PRECISION_MIXED)
    before = ac.get_state()
    path = str(tmp_path / "tune.txt")
    try:
        r1 = solver.autotune(ac, steps=2, cache=path)
        assert not r1["from_cache"] and r1["candidates"] >= 10
        assert 0 < r1["best_ms"] <= r1["default_ms"]
        assert ctx.tuning == r1["best"]
        assert "octree/mixed/L2" in r1["key"]
        # the sample is untouched
        after = ac.get_state()
        for a in range(4):
            assert np.array_equal(before[a], after[a])
        ctx.set_tuning(**solver.default_tuning())
        r2 = solver.autotune(ac, steps=2, cache=path)
        assert r2["from_cache"] and r2["best"] == r1["best"] and r2["candidates"] == 0
        assert ctx.tuning == r1["best"]
        # a case built with the tuned context steps correctly
        ac2 = _channel(ctx, abi.PRECISION_MIXED)
        rep = ac2.step(0.004)
        assert rep.converged and rep.divergence_max <= 1e-8
    finally:
        ctx.set_tuning(**solver.default_tuning())


@pytest.mark.parametrize("tpb", [128, 256])
def test_uniform_threads_per_brick(ctx, tpb):
    """Uniform periodic grid (Taylor-Green 16^3): the smaller CTAs give the
    default's solution to 1e-10 relative."""
    def run(tuning):
        ctx.set_tuning(**tuning)
        try:
            g, cfg = cases.taylor_green(16)
            ns = solver.NSSolver(g, cfg, ctx=ctx)
            ns.set_state(*cases.taylor_green_state(g))
            for _ in range(2):
                rep = ns.step(0.05)
                assert rep.converged
            return ns.u_face(), ns.pressure()
        finally:
            ctx.set_tuning(**solver.default_tuning())
    u0, p0 = run({})
    u1, p1 = run(dict(threads_per_brick=tpb, mg_ctas_per_sm=2048 // tpb))
    assert np.abs(u1 - u0).max() <= 1e-10 * np.abs(u0).max()
    assert np.abs(p1 - p0).max() <= 1e-10 * max(np.abs(p0).max(), 1e-30)


@pytest.mark.parametrize("sweeps", [2, 3])
def test_chebyshev_on_a_singular_uniform_box(ctx, sweeps):
    """Periodic TGV 32^3 (singular: pending means on every level) in the mixed
    form with the Chebyshev smoother against the FP64 form: converged, within
    1e-6, and with no more MG-PCG cycles than Jacobi needs."""
    def run(precision, tuning):
        ctx.set_tuning(**tuning)
        try:
            g, cfg = cases.taylor_green(32)
            ns = solver.NSSolver(g, cfg, precision=precision, ctx=ctx)
            ns.set_state(*cases.taylor_green_state(g))
            reps = [ns.step(0.05) for _ in range(2)]
            assert all(r.converged for r in reps)
            return ns.u_face(), sum(r.poisson_iters for r in reps)
        finally:
            ctx.set_tuning(**solver.default_tuning())
    u64, _ = run(abi.PRECISION_FP64, {})
    uj, it_j = run(abi.PRECISION_MIXED, dict(sweeps=sweeps, smoother=0))
    uc, it_c = run(abi.PRECISION_MIXED, dict(sweeps=sweeps, smoother=1))
    assert np.abs(uc - u64).max() <= 1e-6 * np.abs(u64).max()
    assert it_c <= it_j


def test_mixed_warm_start_tracks_fp64_with_fewer_cycles(ctx):
    """Mixed form with each projection started from the last pressure (scaled
    to the RK stage): within 1e-6 of the FP64 form, converged, and no more
    MG-PCG cycles than starting from zero."""
    def run(tuning, precision=abi.PRECISION_MIXED):
        ctx.set_tuning(**tuning)
        try:
            ac = _channel(ctx, precision)
            cycles = 0
            for _ in range(4):
                rep = ac.step(0.004)
                assert rep.converged and rep.divergence_max <= 1e-8
                cycles += rep.poisson_iters
            return ac.get_state()[:3], cycles
        finally:
            ctx.set_tuning(**solver.default_tuning())
    ref, _ = run({}, abi.PRECISION_FP64)
    cold, n_cold = run(dict(warm_start=0))
    warm, n_warm = run(dict(warm_start=1))
    for a in range(3):
        assert np.abs(warm[a] - ref[a]).max() <= 1e-6 * np.abs(ref[0]).max()
    assert n_warm <= n_cold
