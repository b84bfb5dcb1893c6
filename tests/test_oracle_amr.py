"""Pins the oracle's octree MAC step (oracle/restate_amr.c).

On single-level meshes it must reproduce the uniform restatement (itself
pinned to the compiled reference in test_oracle_pin.py) to 1e-9 relative,
with both pressure solves run to 1e-13; on multi-level meshes it must keep
its invariants (post-projection divergence at the solver tolerance, a
uniform flow through a periodic box untouched, exact mass balance in a closed
box). CPU only.
"""
import numpy as np
import pytest

from amr_helpers import refine_where
from helpers import rel_err
from nabla_b200 import abi, amr, cases

TOL = 1e-9


def lex_index(nx, ny, nz, a, periodic):
    """(level 0, i, j, k) of every reference lexicographic a-face (x fastest);
    on a periodic axis the high face is dropped (the mesh stores one copy)."""
    ex, ey, ez = nx + (a == 0), ny + (a == 1), nz + (a == 2)
    k, j, i = np.meshgrid(np.arange(ez), np.arange(ey), np.arange(ex), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    keep = np.ones(i.size, dtype=bool)
    if periodic:
        n = (nx, ny, nz)[a]
        keep = (i, j, k)[a] < n
    return np.zeros(int(keep.sum()), dtype=np.int32), i[keep], j[keep], k[keep], keep


def cell_index(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.zeros(nx * ny * nz, dtype=np.int32), i.ravel(), j.ravel(), k.ravel()


def single_level_pair(orc, g, cfg, nb0, state, dt):
    geom = amr.make_geom(nb0, (g.dx, g.dy, g.dz), 0, g.faces, origin=g.origin)
    leaves = amr.base_leaves(nb0)
    lev, i, j, k = amr.cell_coords(leaves)
    solid = g.solid[i + g.nx * (j + g.ny * k)]
    A = orc.amr(geom, leaves, cfg, solid=solid)
    per = [g.faces[2 * a]["type"] == abi.BC_PERIODIC for a in range(3)]
    idx = []
    for a in range(3):
        L, fi, fj, fk, keep = lex_index(g.nx, g.ny, g.nz, a, per[a])
        A.set(a, (L, fi, fj, fk), np.asarray(state[a])[keep])
        idx.append(((L, fi, fj, fk), keep))
    ci = cell_index(g.nx, g.ny, g.nz)
    A.set(3, ci, state[3])
    uni = orc.ns(g, cfg)
    uni.set_state(*state)
    uni.step(dt)
    A.step(dt, 1e-13)
    ref = uni.get_state()
    for a in range(3):
        (ix, keep) = idx[a]
        assert rel_err(A.get(a, ix), np.asarray(ref[a])[keep]) < TOL, "uvw"[a]
    assert rel_err(A.get(3, ci), ref[3]) < TOL


def test_single_level_periodic_tgv_matches_uniform_restatement(orc):
    g, cfg = cases.taylor_green(16, poisson_tol=1e-13)
    single_level_pair(orc, g, cfg, (2, 2, 2), cases.taylor_green_state(g), 0.05)


def test_single_level_channel_with_block_matches_uniform_restatement(orc):
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_PARABOLIC, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL, wall_velocity=(0.3, 0, 0)),
             dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = cases.Grid(32, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    g.solid.reshape(16, 16, 32)[6:10, 0:6, 12:18] = 1
    cfg = cases.flow_config(reynolds=200.0, convection=abi.CONV_WENO5, poisson_tol=1e-13)
    rng = np.random.default_rng(4)
    st = [rng.uniform(0.5, 1.0, 33 * 16 * 16), rng.uniform(-0.1, 0.1, 32 * 17 * 16),
          rng.uniform(-0.1, 0.1, 32 * 16 * 17), np.zeros(32 * 16 * 16)]
    w = st[2].reshape(17, 16, 32)
    w[16] = w[0]
    single_level_pair(orc, g, cfg, (4, 2, 2), st, 0.01)


def _periodic_three_level():
    geom = amr.make_geom((2, 2, 2), (0.25, 0.25, 0.25), 2, cases.periodic_faces())
    lv = amr.base_leaves((2, 2, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 1)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 2 and z == 1)
    return geom, lv


def _all_faces(geom, leaves, lmax):
    """(level, i, j, k) of both a-faces of every leaf cell: every stored face
    is among them (the high faces include the fine-side slabs at level
    jumps; on a periodic axis the domain's high face is its low face)."""
    lev, i, j, k = amr.cell_coords(leaves)
    out = []
    for a in range(3):
        hi = [i.copy(), j.copy(), k.copy()]
        hi[a] += 1
        out.append((np.concatenate([lev, lev]), np.concatenate([i, hi[0]]), np.concatenate([j, hi[1]]),
                    np.concatenate([k, hi[2]])))
    return out


def test_multilevel_uniform_flow_is_steady(orc):
    """A uniform velocity through a periodic 3-level box is an exact steady
    state of every rule (WENO of a constant, interpolation, projection)."""
    geom, lv = _periodic_three_level()
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_WENO5, poisson_tol=1e-13)
    A = orc.amr(geom, lv, cfg)
    faces = _all_faces(geom, lv, 2)
    vals = (0.7, -0.2, 0.4)
    for a in range(3):
        A.set(a, faces[a], np.full(faces[a][0].size, vals[a]))
    dmax, _ = A.step(0.01)
    assert dmax < 1e-12
    for a in range(3):
        assert np.abs(A.get(a, faces[a]) - vals[a]).max() < 1e-12


def test_multilevel_projection_and_mass(orc):
    geom = amr.make_geom((2, 2, 2), (1 / 16, 1 / 16, 1 / 16), 2,
                         [dict(type=abi.BC_WALL) for _ in range(5)] +
                         [dict(type=abi.BC_WALL, wall_velocity=(1.0, 0.0, 0.0))])
    lv = amr.base_leaves((2, 2, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 0 and z == 0)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 1 and z == 1)
    cfg = cases.flow_config(reynolds=100.0, convection=abi.CONV_CENTRAL, poisson_tol=1e-13)
    A = orc.amr(geom, lv, cfg)
    faces = _all_faces(geom, lv, 2)
    rng = np.random.default_rng(1)
    for a in range(3):
        A.set(a, faces[a], rng.uniform(-0.3, 0.3, faces[a][0].size))
    dmax, iters = A.step(0.005)
    assert iters > 0
    assert dmax < 1e-9
