"""Seeded synthetic workloads on octree-AMR meshes (host-side set-up only).

``obstacle_channel`` builds the 3-level channel case: [0,4]x[0,1]x[0,1],
base 64x16x16 cells (8x2x2 bricks of 8^3, h0 = 1/16), refined twice
(effective 256x64x64) where the initial vorticity is in its top fifth or a
cell lies within 0.05 of a solid. Uniform inflow U = 1 at x = 0, outlet at
x = 4, no-slip walls on y and z, nu = 1/1000, CFL 0.4. The obstacle is the
union of 6 seeded axis-aligned boxes (sides U[0.05, 0.2], centres x in
U[0.5, 1.5], y, z in U[0.2, 0.8]); a cell is solid when its centre is inside
a box (staircase, as core/src/flow/case.cpp:113-122 marks the cube). The
initial velocity is U plus the curl of a seeded Gaussian random vector
potential whose spectrum peaks at wavenumber 8 (in cycles per unit length),
scaled to an rms perturbation of 0.05.

Refinement works at brick granularity: a leaf is split when the maximum of
|omega| over its cells (sampled on the effective finest grid) is in the top
fifth of that maximum over the leaves of its level, or when any of its cells
is within 0.05 of a box; 2:1 balance is then restored (nb_amr_refine).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import abi, amr, cases


@dataclass
class Modes:
    k: np.ndarray      # [M, 3] angular wave vectors
    c: np.ndarray      # [M, 3] potential amplitudes
    phase: np.ndarray  # [M]
    scale: float = 1.0

    def velocity(self, x, y, z):
        """curl of A = sum_m c_m cos(k_m . x + phase_m): -sin(theta) (k x c)."""
        kc = np.cross(self.k, self.c) * self.scale
        out = [np.zeros_like(x), np.zeros_like(x), np.zeros_like(x)]
        for m in range(self.k.shape[0]):
            s = -np.sin(self.k[m, 0] * x + self.k[m, 1] * y + self.k[m, 2] * z + self.phase[m])
            for d in range(3):
                out[d] += s * kc[m, d]
        return out

    def vorticity_mag(self, x, y, z):
        """|curl curl A| = |-cos(theta) k x (k x c)| summed over modes."""
        kkc = np.cross(self.k, np.cross(self.k, self.c)) * self.scale
        w = [np.zeros_like(x), np.zeros_like(x), np.zeros_like(x)]
        for m in range(self.k.shape[0]):
            cth = -np.cos(self.k[m, 0] * x + self.k[m, 1] * y + self.k[m, 2] * z + self.phase[m])
            for d in range(3):
                w[d] += cth * kkc[m, d]
        return np.sqrt(w[0] ** 2 + w[1] ** 2 + w[2] ** 2)


def random_modes(rng, n_modes=48, k_peak=8.0, k_width=1.5, rms=0.05, sample=None):
    """Gaussian random vector potential: wave numbers |k|/(2 pi) ~ N(k_peak, k_width),
    isotropic directions, Gaussian amplitudes; scaled so the velocity rms over
    `sample` (x, y, z arrays) is `rms`."""
    kmag = 2.0 * np.pi * np.abs(rng.normal(k_peak, k_width, n_modes))
    d = rng.normal(size=(n_modes, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = d * kmag[:, None]
    c = rng.normal(size=(n_modes, 3)) / kmag[:, None]
    phase = rng.uniform(0.0, 2.0 * np.pi, n_modes)
    m = Modes(k, c, phase)
    if sample is not None:
        u = m.velocity(*sample)
        cur = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2))
        m.scale = rms / cur
    return m


def random_boxes(rng, n=6):
    """[n, 2, 3] lower/upper corners."""
    side = rng.uniform(0.05, 0.2, (n, 3))
    centre = np.stack([rng.uniform(0.5, 1.5, n), rng.uniform(0.2, 0.8, n), rng.uniform(0.2, 0.8, n)], axis=1)
    return np.stack([centre - side / 2, centre + side / 2], axis=1)


def inside_boxes(boxes, x, y, z):
    s = np.zeros(x.shape, dtype=bool)
    for lo, hi in boxes:
        s |= (x > lo[0]) & (x < hi[0]) & (y > lo[1]) & (y < hi[1]) & (z > lo[2]) & (z < hi[2])
    return s


def box_distance(boxes, x, y, z):
    d = np.full(x.shape, np.inf)
    for lo, hi in boxes:
        dx = np.maximum(np.maximum(lo[0] - x, 0.0), x - hi[0])
        dy = np.maximum(np.maximum(lo[1] - y, 0.0), y - hi[1])
        dz = np.maximum(np.maximum(lo[2] - z, 0.0), z - hi[2])
        d = np.minimum(d, np.sqrt(dx * dx + dy * dy + dz * dz))
    return d


@dataclass
class AmrWorkload:
    geom: abi.AmrGeom
    leaves: np.ndarray
    solid: np.ndarray  # 512 bytes per leaf, in `leaves` order
    config: abi.FlowConfig
    modes: Modes
    boxes: np.ndarray
    mean_u: float
    description: str

    def initial_state(self, case: amr.AmrCase):
        st = []
        for a in range(3):
            x, y, z = case.face_positions(a)
            u = self.modes.velocity(x, y, z)[a]
            st.append(u + (self.mean_u if a == 0 else 0.0))
        st.append(np.zeros(case.sizes[3]))
        return st


def _leaf_metric(modes, boxes, leaves, h0, lmax, near):
    """Per leaf: max |omega| over its region sampled at the finest cell centres
    (4^3 samples per finest brick-cell block are enough at this resolution:
    every second finest cell), and whether any of its cells is within `near`
    of a box."""
    out_w = np.zeros(len(leaves))
    out_near = np.zeros(len(leaves), dtype=bool)
    for q, (lev, bx, by, bz) in enumerate(leaves):
        h = h0 / (1 << lev)
        n = 8 << (lmax - lev)  # finest cells per brick edge
        hf = h0 / (1 << lmax)
        s = np.arange(0, n, 2) + 0.5
        X, Y, Z = np.meshgrid(bx * 8 * h + s * hf, by * 8 * h + s * hf, bz * 8 * h + s * hf, indexing="ij")
        out_w[q] = modes.vorticity_mag(X.ravel(), Y.ravel(), Z.ravel()).max()
        c = (np.arange(8) + 0.5) * h
        Xc, Yc, Zc = np.meshgrid(bx * 8 * h + c, by * 8 * h + c, bz * 8 * h + c, indexing="ij")
        out_near[q] = (box_distance(boxes, Xc.ravel(), Yc.ravel(), Zc.ravel()) <= near).any()
    return out_w, out_near


def _tgv_vorticity(x, y, z):
    """|curl u| of u = sin x cos y cos z, v = -cos x sin y cos z, w = 0."""
    wx = -np.cos(x) * np.sin(y) * np.sin(z)
    wy = -np.sin(x) * np.cos(y) * np.sin(z)
    wz = 2.0 * np.sin(x) * np.sin(y) * np.cos(z)
    return np.sqrt(wx * wx + wy * wy + wz * wz)


def tgv_face_state(case: amr.AmrCase):
    """The Taylor-Green state u = sin x cos y cos z, v = -cos x sin y cos z, w = 0
    on an octree case's stored faces, p = 0."""
    st = []
    for a in range(3):
        x, y, z = case.face_positions(a)
        if a == 0:
            st.append(np.sin(x) * np.cos(y) * np.cos(z))
        elif a == 1:
            st.append(-np.cos(x) * np.sin(y) * np.cos(z))
        else:
            st.append(np.zeros_like(x))
    st.append(np.zeros(case.sizes[3]))
    return st


@dataclass
class TgvBoxWorkload:
    geom: abi.AmrGeom
    leaves: np.ndarray
    solid: np.ndarray
    config: abi.FlowConfig
    base: int
    levels: int
    n_boxes: int

    def initial_state(self, case: amr.AmrCase):
        return tgv_face_state(case)


def tgv_box_case(seed: int) -> TgvBoxWorkload:
    """One case of the batched workload: the Taylor-Green box [0, 2 pi]^3 on a
    base grid drawn from {16, 24, 32, 48, 64}^3 with 1 to 3 octree levels and
    0 to 6 seeded boxes (sides U[0.05, 0.2] x 2 pi), refined at brick
    granularity where the TGV vorticity is in its top fifth or near a box."""
    rng = np.random.default_rng(1000 + seed)
    base = int(rng.choice([16, 24, 32, 48, 64]))
    levels = int(rng.integers(1, 4))
    n_boxes = int(rng.integers(0, 7))
    L = 2.0 * np.pi
    h0 = L / base
    nb0 = (base // 8,) * 3
    geom = amr.make_geom(nb0, (h0, h0, h0), levels - 1, cases.periodic_faces())
    side = rng.uniform(0.05, 0.2, (n_boxes, 3)) * L
    centre = rng.uniform(0.0, L, (n_boxes, 3))
    boxes = np.stack([centre - side / 2, centre + side / 2], axis=1) if n_boxes else np.zeros((0, 2, 3))
    leaves = amr.base_leaves(nb0)
    for lev in range(levels - 1):
        at = leaves[:, 0] == lev
        w = np.zeros(len(leaves))
        near = np.zeros(len(leaves), dtype=bool)
        for q in np.nonzero(at)[0]:
            lv, bx, by, bz = leaves[q]
            h = h0 / (1 << lv)
            c = (np.arange(8) + 0.5) * h
            X, Y, Z = np.meshgrid(bx * 8 * h + c, by * 8 * h + c, bz * 8 * h + c, indexing="ij")
            w[q] = _tgv_vorticity(X, Y, Z).max()
            if n_boxes:
                near[q] = (box_distance(boxes, X.ravel(), Y.ravel(), Z.ravel()) <= 0.05 * L).any()
        thr = np.percentile(w[at], 80.0)
        flags = (at & ((w > thr) | near)).astype(np.uint8)
        if not flags.any():
            break
        leaves = amr.refine(geom, leaves, flags)
    lev, i, j, k = amr.cell_coords(leaves)
    h = h0 / (2.0 ** lev)
    solid = inside_boxes(boxes, (i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h).astype(np.uint8) if n_boxes else \
        np.zeros(lev.size, dtype=np.uint8)
    cfg = cases.flow_config(reynolds=1600.0, ref_length=1.0, velocity_scale=1.0, cfl=0.4,
                            convection=abi.CONV_WENO5, poisson_tol=1e-10, poisson_max_iters=200)
    return TgvBoxWorkload(geom, leaves, solid, cfg, base, int(leaves[:, 0].max()) + 1, n_boxes)


def tgv_octree(base: int, levels: int = 3):
    """3-level octree of the periodic Taylor-Green box [0, 2 pi]^3 on a base^3
    grid (effective (base * 2^(levels-1))^3), refined at brick granularity
    where the brick-mean TGV vorticity is in its top fifth (the pressure-solve stress
    meshes). Returns (geom, leaves)."""
    L = 2.0 * np.pi
    h0 = L / base
    nb0 = (base // 8,) * 3
    geom = amr.make_geom(nb0, (h0, h0, h0), levels - 1, cases.periodic_faces())
    leaves = amr.base_leaves(nb0)
    c = np.arange(8) + 0.5
    for lev in range(levels - 1):
        at = np.nonzero(leaves[:, 0] == lev)[0]
        h = h0 / (1 << lev)
        b = leaves[at, 1:4].astype(np.float64)
        X = (b[:, 0:1, None, None] * 8 + c[None, :, None, None]) * h
        Y = (b[:, 1:2, None, None] * 8 + c[None, None, :, None]) * h
        Z = (b[:, 2:3, None, None] * 8 + c[None, None, None, :]) * h
        # brick mean of |omega| (the brick maxima of this symmetric field tie)
        w = _tgv_vorticity(X, Y, Z).reshape(len(at), -1).mean(axis=1)
        thr = np.percentile(w, 80.0)
        flags = np.zeros(len(leaves), dtype=np.uint8)
        flags[at[w > thr]] = 1
        leaves = amr.refine(geom, leaves, flags)
    return geom, leaves


CHANNEL_FACES = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
                 dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
                 dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]


def channel_config():
    return cases.flow_config(reynolds=1000.0, ref_length=1.0, velocity_scale=1.0, cfl=0.4,
                             convection=abi.CONV_WENO5, poisson_tol=1e-10, poisson_max_iters=200)


def channel_inputs(seed: int = 0, n_boxes: int = 6):
    """The seeded inputs of the obstacle channel, drawn in a fixed order from
    one stream: the solid boxes, then the random vector potential. Pure numpy
    (no device and no library call), so a CPU-only process can rebuild the
    same case on any grid."""
    rng = np.random.default_rng(seed)
    boxes = random_boxes(rng, n_boxes)
    sx = rng.uniform(0, 4, 20000)
    sy, sz = rng.uniform(0, 1, 20000), rng.uniform(0, 1, 20000)
    modes = random_modes(rng, sample=(sx, sy, sz))
    return boxes, modes


def obstacle_channel(seed: int = 0, lmax: int = 2, n_boxes: int = 6, precision_note: str = "") -> AmrWorkload:
    h0 = 1.0 / 16.0
    nb0 = (8, 2, 2)
    geom = amr.make_geom(nb0, (h0, h0, h0), lmax, CHANNEL_FACES)
    boxes, modes = channel_inputs(seed, n_boxes)
    leaves = amr.base_leaves(nb0)
    for lev in range(lmax):
        w, near = _leaf_metric(modes, boxes, leaves, h0, lmax, 0.05)
        at = leaves[:, 0] == lev
        thr = np.percentile(w[at], 80.0) if at.any() else np.inf
        flags = (at & ((w > thr) | near)).astype(np.uint8)
        if not flags.any():
            break
        leaves = amr.refine(geom, leaves, flags)
    lev, i, j, k = amr.cell_coords(leaves)
    h = h0 / (2.0 ** lev)
    solid = inside_boxes(boxes, (i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h).astype(np.uint8)
    cfg = channel_config()
    nl = np.bincount(leaves[:, 0], minlength=lmax + 1)
    desc = (f"obstacle channel [0,4]x[0,1]^2, octree of 8^3 bricks, base 64x16x16, {lmax + 1} levels "
            f"(effective {64 << lmax}x{16 << lmax}x{16 << lmax}), leaves per level {nl.tolist()}, "
            f"{n_boxes} seeded boxes, inflow U=1 + curl of a k=8 random potential (rms 0.05), "
            f"nu=1/1000, WENO-5, CFL 0.4, MG-PCG to 1e-10, seed {seed}")
    return AmrWorkload(geom, leaves, solid, cfg, modes, boxes, 1.0, desc)


def channel_uniform(seed: int = 0, refine: int = 2, n_boxes: int = 6):
    """The obstacle channel on the uniform grid of its finest level (256x64x64
    cells for refine = 2, h = 1/64): the same seeded boxes (cells whose centre
    is inside are solid) and the same initial velocity sampled on the MAC faces.
    Returns (grid, config, (u, v, w, p)) in the reference's lexicographic
    layout. Pure numpy: no device and no library call."""
    boxes, modes = channel_inputs(seed, n_boxes)
    h = 1.0 / (16 << refine)
    nx, ny, nz = 64 << refine, 16 << refine, 16 << refine
    g = cases.Grid(nx, ny, nz, h, h, h, faces=[dict(f) for f in CHANNEL_FACES])
    zc, yc, xc = np.meshgrid((np.arange(nz) + 0.5) * h, (np.arange(ny) + 0.5) * h, (np.arange(nx) + 0.5) * h,
                             indexing="ij")
    g.solid[:] = inside_boxes(boxes, xc.ravel(), yc.ravel(), zc.ravel()).astype(np.uint8)
    st = []
    for a, (ex, ey, ez) in enumerate([(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]):
        off = [0.5, 0.5, 0.5]
        off[a] = 0.0
        Z, Y, X = np.meshgrid((np.arange(ez) + off[2]) * h, (np.arange(ey) + off[1]) * h,
                              (np.arange(ex) + off[0]) * h, indexing="ij")
        u = modes.velocity(X.ravel(), Y.ravel(), Z.ravel())[a]
        st.append(u + (1.0 if a == 0 else 0.0))
    st.append(np.zeros(g.ncell))
    return g, channel_config(), tuple(st)
