"""Shared helpers of the map-parity tests: carrying a brick tree into the
reference's Octree (core/src/mesh/octree.cpp) and reading its face-neighbour
table back in the library's terms."""
import ctypes as C

import numpy as np


def ref_decode(ref, key):
    x, y, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
    ref.lib.ref_morton_decode(key, C.byref(x), C.byref(y), C.byref(z))
    return x.value, y.value, z.value


def replay_into_reference(ref, nb0, lmax, leaves, extra_levels=0):
    """A reference Octree whose leaves cover the library's `leaves` (level,
    bx, by, bz on a forest of nb0 base bricks): a root cube of 2^k0 base
    bricks (k0 = ceil(log2(max nb0))), maxLevel k0 + lmax + extra_levels;
    library level L is reference level k0 + L + extra_levels when each leaf is
    refined `extra_levels` more times (3 = one reference leaf per cell).
    Every ancestor of a target leaf is refined with refineByMorton, coarsest
    level first, so the reference's own 2:1 face balance never has to add a
    leaf inside the library's domain."""
    k0 = int(np.ceil(np.log2(max(nb0)))) if max(nb0) > 1 else 0
    M = k0 + lmax + extra_levels
    t = ref.octree((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), M)
    if k0:
        t.refine_uniform(k0)
    need = [set() for _ in range(M)]
    for L, bx, by, bz in np.asarray(leaves).tolist():
        s = lmax - L
        a = (bx << s << extra_levels, by << s << extra_levels, bz << s << extra_levels)
        for m in range(k0, k0 + L):  # the leaf's ancestors
            mask = ~((1 << (M - m)) - 1)
            need[m].add(ref.morton_encode(a[0] & mask, a[1] & mask, a[2] & mask))
        size = 1 << (M - (k0 + L))  # the leaf's extent on the finest grid
        for m in range(k0 + L, k0 + L + extra_levels):  # every node inside the leaf above its cells
            step = 1 << (M - m)
            for z in range(a[2], a[2] + size, step):
                for y in range(a[1], a[1] + size, step):
                    for x in range(a[0], a[0] + size, step):
                        need[m].add(ref.morton_encode(x, y, z))
    for m in range(k0, M):
        if not need[m]:
            continue
        keys, lev, _ = t.cells()
        at = dict(zip(keys.tolist(), lev.tolist()))
        for key in sorted(need[m]):
            if at.get(key) == m:
                t.refine_morton(key)
                keys, lev, _ = t.cells()
                at = dict(zip(keys.tolist(), lev.tolist()))
    return t, k0, M


def reference_table(ref, t, domain):
    """The reference's leaves inside `domain` (finest-level extents) as a dict
    key -> (index, level), and a function giving faceNeighbors(i, d) as keys,
    dropping neighbours outside the domain."""
    keys, lev, _ = t.cells()
    keys = keys.tolist()
    lev = lev.tolist()

    def inside(key):
        x, y, z = ref_decode(ref, key)
        return x < domain[0] and y < domain[1] and z < domain[2]

    table = {k: (i, l) for i, (k, l) in enumerate(zip(keys, lev)) if inside(k)}

    def nbrs(i, d):
        return [(keys[q], lev[q]) for q in t.face_neighbors(i, d) if inside(keys[q])]

    return table, nbrs


def compare_tree_with_reference(ref, nb0, lmax, keys, ranked, nbr, cnt):
    """Asserts the library's keys, rank order and face-neighbour table equal the
    reference Octree's on the same tree, integer for integer and in order."""
    t, k0, M = replay_into_reference(ref, nb0, lmax, ranked)
    domain = [nb0[a] << lmax for a in range(3)]
    table, nbrs = reference_table(ref, t, domain)
    ours = {int(k): int(l) + k0 for k, l in zip(keys, ranked[:, 0])}
    theirs = {k: l for k, (_, l) in table.items()}
    assert ours == theirs, "leaf sets differ"
    assert np.all(np.diff(keys.astype(np.uint64).astype(object)) > 0) if len(keys) > 1 else True
    assert [int(k) for k in keys] == sorted(theirs), "rank order differs"
    for r in range(len(keys)):
        i, _ = table[int(keys[r])]
        for d in range(6):
            mine = [(int(keys[q]), int(ranked[q, 0]) + k0) for q in nbr[r, d, :cnt[r, d]]]
            assert mine == nbrs(i, d), (r, d, mine, nbrs(i, d))
    return len(keys)
