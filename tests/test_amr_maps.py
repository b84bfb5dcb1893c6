"""Host-side octree brick maps (integer work, CPU): refinement, 26-neighbour
2:1 balance (the balance rule of Octree::refineByMorton,
core/src/mesh/octree.cpp:325-356, at brick granularity), coverage,
deterministic Morton ranking, and the merging of sibling octets
(Octree::coarsen, core/src/mesh/octree.cpp:393-473)."""
import numpy as np

from amr_helpers import check_balanced, closed_box_geom, refine_where, three_level_leaves, two_level_leaves
from nabla_b200 import abi, amr


def test_refine_one_brick():
    g = closed_box_geom()
    lv = two_level_leaves(g)
    assert len(lv) == 7 + 8
    assert sorted(set(lv[:, 0])) == [0, 1]
    check_balanced(lv, list(g.nb0))


def test_three_levels_balanced():
    g = closed_box_geom()
    lv = three_level_leaves(g)
    assert lv[:, 0].max() == 2
    check_balanced(lv, list(g.nb0))


def test_refine_storm_stays_balanced():
    """Random refine storm (seed 12345, as core/tests/test_octree.cpp:60-77)."""
    g = amr.make_geom((3, 2, 2), (0.1, 0.1, 0.1), 3, [dict(type=abi.BC_WALL) for _ in range(6)])
    rng = np.random.default_rng(12345)
    lv = amr.base_leaves([3, 2, 2])
    for _ in range(6):
        flags = (rng.random(len(lv)) < 0.15).astype(np.uint8)
        lv = amr.refine(g, lv, flags)
        check_balanced(lv, [3, 2, 2])
    assert lv[:, 0].max() == 3


def test_periodic_balance_wraps():
    faces = [dict(type=abi.BC_PERIODIC) for _ in range(6)]
    g = amr.make_geom((4, 2, 2), (0.1, 0.1, 0.1), 2, faces)
    lv = amr.base_leaves([4, 2, 2])
    # refine twice in the corner brick (0,0,0): its periodic neighbours must follow
    lv = amr.refine(g, lv, (lv[:, 1:].sum(axis=1) == 0).astype(np.uint8))
    lv = amr.refine(g, lv, ((lv[:, 0] == 1) & (lv[:, 1:].sum(axis=1) == 0)).astype(np.uint8))
    check_balanced(lv, [4, 2, 2], periodic=(True, True, True))
    # the brick across the periodic x boundary (3,0,0) had to be refined
    assert not ((lv[:, 0] == 0) & (lv[:, 1] == 3) & (lv[:, 2] == 0) & (lv[:, 3] == 0)).any()


def test_no_flags_is_identity_and_deterministic():
    g = closed_box_geom()
    lv = three_level_leaves(g)
    again = amr.refine(g, lv, np.zeros(len(lv), dtype=np.uint8))
    key = lambda a: sorted(map(tuple, a))
    assert key(again) == key(lv)
    assert np.array_equal(three_level_leaves(g), lv)


def test_refine_rejects_bad_leaf_sets():
    g = closed_box_geom()
    lv = amr.base_leaves([2, 2, 2])[:-1]  # hole
    import pytest
    from nabla_b200.solver import NablaError
    with pytest.raises(NablaError):
        amr.refine(g, lv, np.zeros(len(lv), dtype=np.uint8))


def _as_set(leaves):
    return {tuple(int(v) for v in lf) for lf in leaves}


def test_coarsen_undoes_a_uniform_refinement():
    geom = closed_box_geom()
    base = amr.base_leaves(list(geom.nb0))
    fine = amr.refine(geom, base, np.ones(len(base), dtype=np.uint8))
    assert len(fine) == 64
    back = amr.coarsen(geom, fine, np.ones(len(fine), dtype=np.uint8))
    assert _as_set(back) == _as_set(base)


def test_coarsen_keeps_balance():
    geom = closed_box_geom()
    lv = three_level_leaves(geom)  # level-2 leaves inside refined brick (0,0,0)
    # flag every level-1 leaf: the octet under base brick (0,0,0) holds a
    # refined member, so it cannot merge; nothing else is complete
    flags = (lv[:, 0] == 1).astype(np.uint8)
    out = amr.coarsen(geom, lv, flags)
    check_balanced(out, geom.nb0)
    assert _as_set(out) == _as_set(lv)
    # flag the level-2 octet: it merges back, then the level-1 octet can too
    once = amr.coarsen(geom, lv, (lv[:, 0] == 2).astype(np.uint8))
    check_balanced(once, geom.nb0)
    assert int(once[:, 0].max()) == 1
    twice = amr.coarsen(geom, once, np.ones(len(once), dtype=np.uint8))
    assert _as_set(twice) == _as_set(amr.base_leaves(list(geom.nb0)))


def test_coarsen_refuses_a_merge_next_to_two_levels_finer():
    geom = closed_box_geom(nb0=(4, 2, 2))
    lv = amr.base_leaves(list(geom.nb0))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 0 and x in (1, 2))
    lv = refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 4 and y == 0 and z == 0)
    check_balanced(lv, geom.nb0)
    # the level-1 octet of base brick 1 touches the level-2 leaves inside brick 2
    out = amr.coarsen(geom, lv, ((lv[:, 0] == 1) & (lv[:, 1] < 4)).astype(np.uint8))
    check_balanced(out, geom.nb0)
    assert (1, 2, 0, 0) in _as_set(out)  # still refined
