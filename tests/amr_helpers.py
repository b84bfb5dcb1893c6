"""Helpers shared by the octree-AMR tests."""
import numpy as np

from nabla_b200 import abi, amr


def closed_box_geom(nb0=(2, 2, 2), lmax=2, h0=1.0 / 16):
    return amr.make_geom(nb0, (h0, h0, h0), lmax, [dict(type=abi.BC_WALL) for _ in range(6)])


def refine_where(geom, leaves, pred):
    flags = np.array([1 if pred(*lf) else 0 for lf in leaves], dtype=np.uint8)
    return amr.refine(geom, leaves, flags)


def two_level_leaves(geom):
    """Base bricks plus one refined base brick (brick (0,0,0))."""
    lv = amr.base_leaves(list(geom.nb0))
    return refine_where(geom, lv, lambda L, x, y, z: L == 0 and x == 0 and y == 0 and z == 0)


def three_level_leaves(geom):
    lv = two_level_leaves(geom)
    return refine_where(geom, lv, lambda L, x, y, z: L == 1 and x == 1 and y == 1 and z == 1)


def leaf_extents(leaves, nb0):
    """Integer extents of each leaf on the finest grid (units of finest brick)."""
    lmax = int(leaves[:, 0].max())
    s = 1 << (lmax - leaves[:, 0])
    lo = leaves[:, 1:4] * s[:, None]
    return lo, lo + s[:, None], lmax


def check_balanced(leaves, nb0, periodic=(False, False, False)):
    """26-neighbour 2:1 balance and exact coverage (slow reference check)."""
    lo, hi, lmax = leaf_extents(leaves, nb0)
    dims = np.array(nb0) << lmax
    owner = -np.ones(tuple(dims[::-1]), dtype=np.int64)
    for q in range(len(leaves)):
        owner[lo[q, 2]:hi[q, 2], lo[q, 1]:hi[q, 1], lo[q, 0]:hi[q, 0]] = q
    assert (owner >= 0).all(), "coverage"
    lev = leaves[:, 0]
    for axis in range(3):
        for shift in (1, -1):
            nbr = np.roll(owner, shift, axis=2 - axis)
            if not periodic[axis]:
                sl = [slice(None)] * 3
                sl[2 - axis] = slice(0, 1) if shift == 1 else slice(-1, None)
                nbr[tuple(sl)] = owner[tuple(sl)]
            d = np.abs(lev[owner] - lev[nbr])
            assert d.max() <= 1
    # edges / corners via diagonal shifts
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dx, dy, dz) == (0, 0, 0):
                    continue
                nbr = np.roll(owner, (dz, dy, dx), axis=(0, 1, 2))
                valid = np.ones_like(owner, dtype=bool)
                for a, dd in ((2, dx), (1, dy), (0, dz)):
                    if dd == 0 or periodic[2 - a]:
                        continue
                    sl = [slice(None)] * 3
                    sl[a] = slice(0, 1) if dd == 1 else slice(-1, None)
                    valid[tuple(sl)] = False
                d = np.abs(lev[owner] - lev[nbr])[valid]
                assert d.max() <= 1
