"""GPU parity of the composite (octree-AMR) pressure operator and its MG-PCG
solve, through the C ABI.

The operator is pinned against the reference's own OctreePoisson::applyA
(core/src/flow/octree_poisson.cpp:64-85) on brick-aligned trees built with
the reference's refineUniform/refineBox: ours is per unit volume, so
(ours * V) must equal the reference to 1e-12 relative (same neighbours, same
coefficients; only the association of the coefficient arithmetic differs).
"""
import math

import numpy as np
import pytest

from amr_helpers import closed_box_geom, three_level_leaves, two_level_leaves
from helpers import rel_err
from nabla_b200 import abi, amr, cases, solver

pytestmark = pytest.mark.gpu
MAXLEVEL = 8


def morton_decode(keys):
    keys = np.asarray(keys, dtype=np.uint64)
    out = []
    for axis in range(3):
        v = np.zeros(keys.shape, dtype=np.int64)
        for b in range(21):
            v |= ((keys >> np.uint64(3 * b + axis)) & np.uint64(1)).astype(np.int64) << b
        out.append(v)
    return out


def reference_tree(ref, leaves, nb0, h0):
    base = int(round(math.log2(8 * nb0)))
    t = ref.octree((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), MAXLEVEL)
    t.refine_uniform(base)
    lmax = int(leaves[:, 0].max())
    for L in range(lmax):
        par = sorted({(int(f[1]) >> (int(f[0]) - L), int(f[2]) >> (int(f[0]) - L), int(f[3]) >> (int(f[0]) - L))
                      for f in leaves if f[0] > L})
        size = 8 * h0 / 2 ** L
        for bx, by, bz in par:
            lo = (bx * size, by * size, bz * size)
            t.refine_box(lo, (lo[0] + size, lo[1] + size, lo[2] + size), 1)
    return t, base


def map_reference(t, base, mesh):
    keys, lev, _ = t.cells()
    ax, ay, az = morton_decode(keys)
    L = lev.astype(np.int64) - base
    sh = MAXLEVEL - lev.astype(np.int64)
    i, j, k = ax >> sh, ay >> sh, az >> sh
    rank = {(int(f[0]), int(f[1]), int(f[2]), int(f[3])): r for r, f in enumerate(mesh.leaves)}
    idx = np.array([rank[(int(l), int(a >> 3), int(b >> 3), int(c >> 3))] * 512 + (int(c & 7) * 64 + int(b & 7) * 8 + int(a & 7))
                    for l, a, b, c in zip(L, i, j, k)])
    return idx, L


@pytest.mark.parametrize("which", ["two", "three"])
def test_operator_matches_reference_octree_poisson(ctx, ref, which):
    g = closed_box_geom()
    leaves = two_level_leaves(g) if which == "two" else three_level_leaves(g)
    mesh = amr.AmrMesh(g, leaves, ctx=ctx)
    t, base = reference_tree(ref, mesh.leaves, 2, 1.0 / 16)
    idx, L = map_reference(t, base, mesh)
    assert len(idx) == mesh.ncell and len(set(idx)) == mesh.ncell, "leaf sets differ"
    x_ref = np.random.default_rng(2024).uniform(-1, 1, len(idx))
    x = np.zeros(mesh.ncell)
    x[idx] = x_ref
    out_ref = t.apply_a(x_ref)
    V = (1.0 / (16 * 2.0 ** L)) ** 3
    got = mesh.apply_a(x)[idx] * V
    assert rel_err(got, out_ref) < 1e-12


def test_operator_with_non_fluid_cells_matches_reference(ctx, ref):
    g = closed_box_geom()
    leaves = three_level_leaves(g)
    m0 = amr.AmrMesh(g, leaves, ctx=ctx)
    t, base = reference_tree(ref, m0.leaves, 2, 1.0 / 16)
    idx, L = map_reference(t, base, m0)
    rng = np.random.default_rng(7)
    mask = rng.random(len(idx)) < 0.1
    for c in np.flatnonzero(mask):
        t.set_mask(int(c), 2)  # InsideSolid
    solid = np.zeros(m0.ncell, dtype=np.uint8)
    solid[idx[mask]] = 1
    mesh = amr.AmrMesh(g, m0.leaves, solid=solid, ctx=ctx)
    x_ref = rng.uniform(-1, 1, len(idx))
    x = np.zeros(mesh.ncell)
    x[idx] = x_ref
    out_ref = t.apply_a(x_ref)
    V = (1.0 / (16 * 2.0 ** L)) ** 3
    got = mesh.apply_a(x)[idx]
    got = np.where(mask, got, got * V)  # identity rows are not volume scaled
    assert rel_err(got, out_ref) < 1e-12


def test_operator_symmetric_and_conservative(ctx):
    g = closed_box_geom()
    mesh = amr.AmrMesh(g, three_level_leaves(g), ctx=ctx)
    hx, hy, hz = mesh.cell_size()
    V = hx * hy * hz
    rng = np.random.default_rng(3)
    a, b = rng.uniform(-1, 1, mesh.ncell), rng.uniform(-1, 1, mesh.ncell)
    Aa, Ab = mesh.apply_a(a), mesh.apply_a(b)
    assert abs(np.sum(V * a * Ab) - np.sum(V * b * Aa)) < 1e-10 * abs(np.sum(V * a * Ab))
    assert abs(np.sum(V * Aa)) < 1e-9 * (1 + np.abs(V * Aa).max())


def test_single_level_mesh_matches_uniform_operator(ctx):
    faces = [dict(type=abi.BC_INLET), dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = amr.make_geom((4, 2, 2), (1 / 16, 1 / 16, 1 / 16), 0, faces)
    mesh = amr.AmrMesh(g, amr.base_leaves([4, 2, 2]), ctx=ctx)
    grid = cases.Grid(32, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    lev, i, j, k = amr.cell_coords(mesh.leaves)
    lex = i + 32 * (j + 16 * k)
    x = np.random.default_rng(5).uniform(-1, 1, mesh.ncell)
    xl = np.zeros(grid.ncell)
    xl[lex] = x
    uni = solver.apply_a(grid, xl, ctx)
    assert rel_err(mesh.apply_a(x), uni[lex]) < 1e-14
    b = np.random.default_rng(6).standard_normal(mesh.ncell)
    bl = np.zeros(grid.ncell)
    bl[lex] = b
    xm, rm = mesh.solve(b, 1e-10, 100)
    xu, ru = solver.MgPoisson(1e-10, 100, ctx=ctx).solve(grid, bl)
    assert rm.iterations == ru.iterations
    assert rel_err(xm, xu[lex]) < 1e-12


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_manufactured_solution_across_level_jumps(ctx, precision):
    """core/tests/test_octree_poisson.cpp:67-97 on the brick mesh: b = A p_exact
    for p = cos(pi x) cos(pi y) cos(pi z); the solve recovers p up to a constant."""
    g = closed_box_geom()
    mesh = amr.AmrMesh(g, three_level_leaves(g), ctx=ctx)
    cx, cy, cz = mesh.cell_centers()
    p = np.cos(np.pi * cx) * np.cos(np.pi * cy) * np.cos(np.pi * cz)
    b = mesh.apply_a(p)
    x, rep = mesh.solve(b, 1e-10, 200, precision=precision)
    assert rep.converged and rep.residual < 1e-8
    assert rep.iterations <= 40
    hx, hy, hz = mesh.cell_size()
    V = hx * hy * hz
    e = (x - np.sum(V * x) / V.sum()) - (p - np.sum(V * p) / V.sum())
    assert np.sqrt(np.sum(V * e * e) / V.sum()) < 1e-6
