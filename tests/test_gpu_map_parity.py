"""Bit-exact parity of the device-built octree maps (nb_amr_build_maps:
Morton keys, a device sort for the rank order, face neighbours by binary
search) with the library's host tree and with the reference's Octree.

* On the library's own meshes (the obstacle channel, a periodic Taylor-Green
  box, a refinement storm): the device keys, rank order and face-neighbour
  table equal the host tree's (nb_amr_tree_maps) and the mesh's own
  (nb_amr_mesh_maps), integer for integer.
* On trees the reference builds itself (refineUniform, refineBox,
  refineByMorton, coarsen; 2:1 across faces only, which the device builder
  accepts): the device table equals Octree::faceNeighbors
  (core/src/mesh/octree.cpp:229-283) for every leaf and face, in order.
* Coarse-fine couplings of the composite operator (nb_amr_mesh_couplings) at
  cell granularity: every cell's coupled neighbours are exactly the cells the
  reference's Octree (refined to one leaf per cell) lists across level jumps,
  with the per-unit-volume coefficients of the octree face rule
  (core/src/flow/octree_poisson.cpp:24-32): 1/(1.5 h^2) to a coarser cell,
  1/(3 h^2) to each finer one.
"""
import numpy as np
import pytest

from amr_helpers import refine_where
from map_helpers import ref_decode, replay_into_reference
from nabla_b200 import abi, amr, workloads

pytestmark = pytest.mark.gpu


def _same_maps(ctx, geom, leaves):
    dk, order, dn, dc = amr.build_maps(geom, leaves, ctx)
    hk, ranked, hn, hc = amr.tree_maps(geom, leaves)
    assert np.array_equal(dk, hk)
    assert np.array_equal(np.asarray(leaves)[order], ranked)
    assert np.array_equal(dc, hc)
    assert np.array_equal(dn, hn)
    return ranked, hk, hn, hc


def test_device_maps_equal_host_maps_on_library_meshes(ctx):
    w = workloads.obstacle_channel(0)
    ranked, keys, nbr, cnt = _same_maps(ctx, w.geom, w.leaves[::-1].copy())
    mesh = amr.AmrMesh(w.geom, w.leaves, solid=w.solid, ctx=ctx)
    mk, mn, mc = mesh.maps()
    assert np.array_equal(mk, keys) and np.array_equal(mn, nbr) and np.array_equal(mc, cnt)
    assert np.array_equal(mesh.leaves, ranked)
    mesh.close()
    t = workloads.tgv_box_case(3)  # periodic: neighbours wrap
    perm = np.random.default_rng(0).permutation(len(t.leaves))
    _same_maps(ctx, t.geom, t.leaves[perm])
    g = amr.make_geom((3, 2, 2), (0.1, 0.1, 0.1), 3, [dict(type=abi.BC_WALL) for _ in range(6)])
    rng = np.random.default_rng(12345)
    lv = amr.base_leaves([3, 2, 2])
    for _ in range(5):
        lv = amr.refine(g, lv, (rng.random(len(lv)) < 0.15).astype(np.uint8))
    _same_maps(ctx, g, lv)


def test_device_maps_equal_reference_on_reference_built_trees(ctx, ref):
    M = 5
    t = ref.octree((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), M)
    t.refine_uniform(2)
    t.refine_box((0.2, 0.3, 0.1), (0.45, 0.6, 0.5), 2)
    rng = np.random.default_rng(7)
    for _ in range(40):
        keys, lev, _ = t.cells()
        i = int(rng.integers(len(keys)))
        if lev[i] < M:
            t.refine_morton(int(keys[i]))
    keys, lev, _ = t.cells()
    keys, lev = [int(k) for k in keys], [int(v) for v in lev]
    for i in range(0, len(keys), 8):
        if lev[i] > 2:
            t.coarsen(keys[i] & ~((1 << (3 * (M - lev[i] + 1))) - 1), lev[i] - 1)
    assert t.is_balanced()
    keys, lev, _ = t.cells()
    keys, lev = keys.tolist(), lev.tolist()
    leaves = np.array([[l] + [c >> (M - l) for c in ref_decode(ref, k)] for k, l in zip(keys, lev)],
                      dtype=np.int32)
    geom = amr.make_geom((1, 1, 1), (1.0, 1.0, 1.0), M, [dict(type=abi.BC_WALL) for _ in range(6)])
    dk, order, dn, dc = amr.build_maps(geom, leaves, ctx)
    assert [int(k) for k in dk] == sorted(keys)
    for r in range(len(dk)):
        i = int(order[r])
        assert int(dk[r]) == keys[i]
        for d in range(6):
            mine = [int(order[q]) for q in dn[r, d, :dc[r, d]]]
            assert mine == t.face_neighbors(i, d), (r, d)


def test_coarse_fine_couplings_match_reference_cell_tree(ctx, ref):
    geom = amr.make_geom((1, 1, 1), (1.0 / 8, 1.0 / 8, 1.0 / 8), 2, [dict(type=abi.BC_WALL) for _ in range(6)])
    lv = refine_where(geom, amr.base_leaves((1, 1, 1)), lambda L, x, y, z: True)
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 0 and z == 1)
    mesh = amr.AmrMesh(geom, lv, ctx=ctx)
    off, cnbr, coef = mesh.couplings()
    ranked = mesh.leaves
    t, k0, M = replay_into_reference(ref, [1, 1, 1], 2, ranked, extra_levels=3)
    keys, lev, _ = t.cells()
    keys, lev = keys.tolist(), lev.tolist()
    index = {k: i for i, k in enumerate(keys)}
    assert len(keys) == mesh.ncell

    def cell_key(c):
        r, l = divmod(int(c), 512)
        L, bx, by, bz = ranked[r].tolist()
        s = 2 - L
        ijk = ((bx * 8 + (l & 7)) << s, (by * 8 + ((l >> 3) & 7)) << s, (bz * 8 + (l >> 6)) << s)
        return ref.morton_encode(*ijk), L

    checked = 0
    for c in range(mesh.ncell):
        key, L = cell_key(c)
        i = index[key]
        assert lev[i] == L + 3
        theirs = sorted(keys[q] for d in range(6) for q in t.face_neighbors(i, d) if lev[q] != lev[i])
        mine = sorted(cell_key(n)[0] for n in cnbr[off[c]:off[c + 1]])
        assert mine == theirs, c
        h2 = (1.0 / 8 / 2 ** L) ** 2
        for n, cf in zip(cnbr[off[c]:off[c + 1]], coef[off[c]:off[c + 1]]):
            want = 1.0 / (1.5 * h2) if cell_key(n)[1] < L else 1.0 / (3.0 * h2)
            assert cf == pytest.approx(want, rel=1e-14)
        checked += off[c + 1] - off[c]
    assert checked > 0
    mesh.close()
