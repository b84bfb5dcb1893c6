"""Bit-exact parity of the library's integer maps with the reference's Octree
(CPU: the library's host tree through nb_amr_tree_maps, the compiled
reference through oracle/_ref).

* Morton keys: the library's encoder (nb_morton.h through nb_morton_encode /
  nb_morton_decode) against the reference's mortonEncode on 20,000 seeded
  triples over the full 21-bit range, the corner values and the per-axis
  bits (core/tests/test_morton.cpp:10-39).
* Rank order and face neighbours: the library's tree, carried into the
  reference's Octree by refineByMorton (core/src/mesh/octree.cpp:325-356),
  gives the same leaf set, the same ascending-key order and, for every leaf
  and face, the same neighbours in the same order as Octree::faceNeighbors
  (octree.cpp:229-283): the neighbour-count case of
  core/tests/test_octree.cpp:136-170, a seeded refinement storm (seed 12345,
  as test_octree.cpp:60-77) and the 3-level obstacle channel mesh.
"""
import numpy as np

from map_helpers import compare_tree_with_reference
from nabla_b200 import abi, amr, workloads


def test_morton_known_answers_on_the_library_encoder(ref):
    assert amr.morton_encode(1, 0, 0) == 0x1
    assert amr.morton_encode(0, 1, 0) == 0x2
    assert amr.morton_encode(0, 0, 1) == 0x4
    top = (1 << 21) - 1
    assert amr.morton_decode(amr.morton_encode(0, 0, 0)) == (0, 0, 0)
    assert amr.morton_decode(amr.morton_encode(top, top, top)) == (top, top, top)
    rng = np.random.default_rng(0xC0FFEE)
    xyz = rng.integers(0, top + 1, size=(20000, 3))
    for x, y, z in xyz.tolist():
        k = amr.morton_encode(x, y, z)
        assert k == ref.morton_encode(x, y, z)
        assert amr.morton_decode(k) == (x, y, z)


def _walls():
    return [dict(type=abi.BC_WALL) for _ in range(6)]


def test_neighbour_counts_across_a_level_jump_match_reference(ref):
    """test_octree.cpp:136-170 at brick granularity: a 4x4x4 tree with one
    interior leaf refined; the coarse east neighbour sees 4 finer ones."""
    g = amr.make_geom((1, 1, 1), (1.0, 1.0, 1.0), 3, _walls())
    lv = amr.base_leaves((1, 1, 1))
    lv = amr.refine(g, lv, np.ones(len(lv), dtype=np.uint8))
    lv = amr.refine(g, lv, np.ones(len(lv), dtype=np.uint8))
    lv = amr.refine(g, lv, ((lv[:, 1] == 1) & (lv[:, 2] == 1) & (lv[:, 3] == 1)).astype(np.uint8))
    keys, ranked, nbr, cnt = amr.tree_maps(g, lv)
    east = [r for r in range(len(ranked)) if tuple(ranked[r]) == (2, 2, 1, 1)][0]
    assert cnt[east, 0] == 4 and set(cnt[east, 1:].tolist()) == {1}
    compare_tree_with_reference(ref, [1, 1, 1], 3, keys, ranked, nbr, cnt)


def test_refinement_storm_matches_reference(ref):
    g = amr.make_geom((1, 1, 1), (1.0, 1.0, 1.0), 4, _walls())
    rng = np.random.default_rng(12345)
    lv = amr.refine(g, amr.base_leaves((1, 1, 1)), np.ones(1, dtype=np.uint8))
    for _ in range(4):
        lv = amr.refine(g, lv, (rng.random(len(lv)) < 0.2).astype(np.uint8))
    assert lv[:, 0].max() >= 3
    n = compare_tree_with_reference(ref, [1, 1, 1], 4, *amr.tree_maps(g, lv))
    assert n == len(lv)


def test_channel_mesh_maps_match_reference(ref):
    w = workloads.obstacle_channel(0)
    keys, ranked, nbr, cnt = amr.tree_maps(w.geom, w.leaves)
    assert len(keys) == 508
    compare_tree_with_reference(ref, list(w.geom.nb0), w.geom.lmax, keys, ranked, nbr, cnt)
