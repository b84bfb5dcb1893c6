"""The adaptive control plane's flow seam (SolverBackend,
core/include/nabla/adaptive/run.hpp:11-32) on the GPU.

CudaSolverBackend (nabla-ai_b200/integration/nabla_adaptive_cuda.hpp), built
into the reference-side test library, is stepped beside the reference's own
NSSolver on the wall-mounted-cube baseline the adaptive run uses; its sample()
must return what BaselineBackend::sample (core/src/adaptive/run.cpp:49-62)
returns, within 1e-10 relative, and sampleMany / sampleFlowCuda must agree
with sample() exactly. nb_case_sample on octree cases: a single-level mesh
samples exactly like the uniform case with the same state, and on a 2-level
mesh every cell-centre sample is the average of the cell's stored faces."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, cases, solver
from test_gpu_amr_step import lex_maps

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin():
    import oracle
    return oracle.Dropin()


def _points(g, n, seed):
    rng = np.random.default_rng(seed)
    ext = np.array([g.nx * g.dx, g.ny * g.dy, g.nz * g.dz])
    pts = rng.uniform(0.0, 1.0, (n, 3)) * ext + np.asarray(g.origin)
    out = rng.uniform(-0.2, 1.2, (16, 3)) * ext + np.asarray(g.origin)  # clamped into the grid
    return np.vstack([pts, out])


def test_cuda_solver_backend_matches_baseline(dropin):
    g, cfg = cases.wall_mounted_cube(4, 500.0)
    pts = _points(g, 400, 1)
    one, many, ref, tele, ref_tele, tree_err = dropin.backend(g, cfg, 3, pts)
    assert np.array_equal(one, many)
    for c in range(4):
        scale = max(np.abs(ref[c]).max(), 1e-30)
        assert np.abs(one[c] - ref[c]).max() <= 1e-10 * scale, c
    assert tele[0] == pytest.approx(ref_tele[0], rel=1e-12)  # t
    assert tele[1] == pytest.approx(ref_tele[1], rel=1e-12)  # dt
    assert tele[3] == pytest.approx(ref_tele[3], rel=1e-8)   # momentum residual
    assert tele[5] == ref_tele[5]                            # poisson iterations
    assert tree_err == 0.0


def _closed_box():
    faces = [dict(type=abi.BC_WALL) for _ in range(6)]
    faces[3] = dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))
    g = cases.Grid(16, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_CENTRAL, poisson_tol=1e-10)
    return g, cfg


def test_single_level_octree_samples_like_uniform(ctx):
    g, cfg = _closed_box()
    st = cases.random_state(g, 5, amp=0.5)
    uni = solver.NSSolver(g, cfg, ctx=ctx)
    uni.set_state(*st)
    geom = amr.make_geom((2, 2, 2), (g.dx, g.dy, g.dz), 0, g.faces, origin=g.origin)
    mesh = amr.AmrMesh(geom, amr.base_leaves((2, 2, 2)), ctx=ctx)
    ac = amr.AmrCase(mesh, cfg)
    ac.set_state(*[np.asarray(s)[m] for s, m in zip(st, lex_maps(ac, g))])
    pts = _points(g, 500, 2)
    for c in range(4):
        assert np.array_equal(ac.sample(c, pts), uni.sample(c, pts)), c


def test_two_level_octree_cell_centre_samples(ctx):
    g, cfg = _closed_box()
    geom = amr.make_geom((2, 2, 2), (g.dx, g.dy, g.dz), 1, g.faces, origin=g.origin)
    lv = amr.base_leaves((2, 2, 2))
    lv = amr.refine(geom, lv, (lv[:, 1] == 0).astype(np.uint8))
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    ac = amr.AmrCase(mesh, cfg)
    rng = np.random.default_rng(6)
    ac.set_state(*[rng.uniform(-1, 1, n) for n in ac.sizes])
    st = ac.get_state()
    x, y, z = mesh.cell_centers()
    pts = np.stack([x, y, z], axis=1)
    ncell = mesh.ncell
    loc = np.arange(ncell) % 512
    cell_loc = (loc & 7, (loc >> 3) & 7, loc >> 6)
    for a, stride in enumerate((1, 8, 64)):
        got = ac.sample(a, pts)
        inner = cell_loc[a] < 7  # the high face is the next cell's low face
        idx = np.arange(ncell)[inner]
        assert np.array_equal(got[inner], 0.5 * (st[a][idx] + st[a][idx + stride]))
    assert np.array_equal(ac.sample(3, pts), st[3])
