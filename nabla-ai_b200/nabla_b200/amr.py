"""Octree-AMR brick meshes over the C ABI (nb_amr_*).

A leaf is (level, bx, by, bz): a brick of 8x8x8 cells at octree level
`level`, brick coordinates in that level's brick grid. Cell arrays over a
mesh are nleaf*512 float64 in the mesh's rank order (Morton order of the
leaf anchors on the finest level), x fastest inside a brick.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .solver import Context, NablaError, Report, default_context


def make_geom(nb0, h0, lmax, faces, origin=(0.0, 0.0, 0.0)) -> abi.AmrGeom:
    g = abi.AmrGeom()
    g.nb0[:] = list(nb0)
    g.h0[:] = list(h0)
    g.origin[:] = list(origin)
    g.lmax = lmax
    for f in range(6):
        spec = faces[f]
        g.face[f].type = spec.get("type", abi.BC_WALL)
        g.face[f].profile = spec.get("profile", abi.PROFILE_UNIFORM)
        g.face[f].inlet_axis = spec.get("inlet_axis", 0)
        g.face[f].inlet_speed = spec.get("inlet_speed", 0.0)
        g.face[f].wall_velocity[:] = list(spec.get("wall_velocity", (0.0, 0.0, 0.0)))
    return g


def base_leaves(nb0) -> np.ndarray:
    z, y, x = np.meshgrid(np.arange(nb0[2]), np.arange(nb0[1]), np.arange(nb0[0]), indexing="ij")
    n = x.size
    return np.stack([np.zeros(n, dtype=np.int32), x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.int32)


def refine(geom: abi.AmrGeom, leaves: np.ndarray, flags: np.ndarray) -> np.ndarray:
    """Split flagged leaves and restore 26-neighbour 2:1 balance (host maps)."""
    lib = abi.load()
    leaves = np.ascontiguousarray(leaves, dtype=np.int32)
    flags = np.ascontiguousarray(flags, dtype=np.uint8)
    n = leaves.shape[0]
    need = C.c_int64()
    cap = max(8 * n, 64)
    while True:
        out = np.zeros((cap, 4), dtype=np.int32)
        st = lib.nb_amr_refine(C.byref(geom), leaves.ctypes.data_as(C.POINTER(C.c_int32)), n,
                               flags.ctypes.data_as(C.POINTER(C.c_uint8)),
                               out.ctypes.data_as(C.POINTER(C.c_int32)), cap, C.byref(need))
        if st == abi.NB_OK:
            return out[:need.value].copy()
        if need.value > cap:
            cap = need.value
            continue
        raise NablaError(st, "nb_amr_refine failed")


def refine_device(geom: abi.AmrGeom, leaves: np.ndarray, flags: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    """The same refinement as refine(), computed on the device (nb_amr_refine_device);
    the new leaves come back in rank order."""
    ctx = ctx or default_context()
    leaves = np.ascontiguousarray(leaves, dtype=np.int32)
    flags = np.ascontiguousarray(flags, dtype=np.uint8)
    n = leaves.shape[0]
    need = C.c_int64()
    cap = max(8 * n, 64)
    out = np.zeros((cap, 4), dtype=np.int32)
    ctx.check(ctx.lib.nb_amr_refine_device(ctx.h, C.byref(geom), leaves.ctypes.data_as(C.POINTER(C.c_int32)), n,
                                           flags.ctypes.data_as(C.POINTER(C.c_uint8)),
                                           out.ctypes.data_as(C.POINTER(C.c_int32)), cap, C.byref(need)),
              "nb_amr_refine_device")
    return out[:need.value].copy()


def coarsen(geom: abi.AmrGeom, leaves: np.ndarray, flags: np.ndarray) -> np.ndarray:
    """Merge complete flagged sibling octets into their parents where the 2:1
    balance allows (nb_amr_coarsen)."""
    lib = abi.load()
    leaves = np.ascontiguousarray(leaves, dtype=np.int32)
    flags = np.ascontiguousarray(flags, dtype=np.uint8)
    n = leaves.shape[0]
    need = C.c_int64()
    out = np.zeros((n, 4), dtype=np.int32)
    st = lib.nb_amr_coarsen(C.byref(geom), leaves.ctypes.data_as(C.POINTER(C.c_int32)), n,
                            flags.ctypes.data_as(C.POINTER(C.c_uint8)), out.ctypes.data_as(C.POINTER(C.c_int32)),
                            n, C.byref(need))
    if st != abi.NB_OK:
        raise ValueError("nb_amr_coarsen rejected the leaf list")
    return out[:need.value].copy()


def morton_encode(x: int, y: int, z: int) -> int:
    """The library's Morton key (nb_morton.h through the C ABI)."""
    return int(abi.load().nb_morton_encode(x, y, z))


def morton_decode(key: int):
    x, y, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
    abi.load().nb_morton_decode(key, C.byref(x), C.byref(y), C.byref(z))
    return x.value, y.value, z.value


def _map_arrays(n):
    return (np.zeros(n, dtype=np.uint64), np.zeros((n, 4), dtype=np.int32), np.zeros((n, 6, 4), dtype=np.int32),
            np.zeros((n, 6), dtype=np.int32))


def tree_maps(geom: abi.AmrGeom, leaves: np.ndarray):
    """Host-only: (keys, leaves in rank order, face-neighbour ranks [n,6,4], counts [n,6])
    of the tree nb_amr_mesh_create builds from `leaves` (nb_amr_tree_maps)."""
    leaves = np.ascontiguousarray(leaves, dtype=np.int32)
    n = leaves.shape[0]
    keys, ranked, nbr, cnt = _map_arrays(n)
    I32 = C.POINTER(C.c_int32)
    st = abi.load().nb_amr_tree_maps(C.byref(geom), leaves.ctypes.data_as(I32), n,
                                     keys.ctypes.data_as(C.POINTER(C.c_uint64)), ranked.ctypes.data_as(I32),
                                     nbr.ctypes.data_as(I32), cnt.ctypes.data_as(I32))
    if st != abi.NB_OK:
        raise NablaError(st, "nb_amr_tree_maps rejected the leaf list")
    return keys, ranked, nbr, cnt


def build_maps(geom: abi.AmrGeom, leaves: np.ndarray, ctx: Context | None = None):
    """Device-built (keys, order, face-neighbour ranks [n,6,4], counts [n,6]) of any
    leaf list (nb_amr_build_maps); order[r] is the input position of rank r."""
    ctx = ctx or default_context()
    leaves = np.ascontiguousarray(leaves, dtype=np.int32)
    n = leaves.shape[0]
    keys, _, nbr, cnt = _map_arrays(n)
    order = np.zeros(n, dtype=np.int32)
    I32 = C.POINTER(C.c_int32)
    ctx.check(ctx.lib.nb_amr_build_maps(ctx.h, C.byref(geom), leaves.ctypes.data_as(I32), n,
                                        keys.ctypes.data_as(C.POINTER(C.c_uint64)), order.ctypes.data_as(I32),
                                        nbr.ctypes.data_as(I32), cnt.ctypes.data_as(I32)), "nb_amr_build_maps")
    return keys, order, nbr, cnt


def cell_coords(leaves: np.ndarray):
    """(level, i, j, k) of every cell, leaves x 512, in array order."""
    l = np.arange(512)
    li, lj, lk = l & 7, (l >> 3) & 7, l >> 6
    lev = np.repeat(leaves[:, 0], 512)
    i = (leaves[:, 1:2] * 8 + li[None, :]).ravel()
    j = (leaves[:, 2:3] * 8 + lj[None, :]).ravel()
    k = (leaves[:, 3:4] * 8 + lk[None, :]).ravel()
    return lev, i, j, k


class AmrMesh:
    def __init__(self, geom: abi.AmrGeom, leaves: np.ndarray, solid: np.ndarray | None = None,
                 ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.geom = geom
        leaves = np.ascontiguousarray(leaves, dtype=np.int32)
        sp = None
        if solid is not None:
            solid = np.ascontiguousarray(solid, dtype=np.uint8)
            sp = solid.ctypes.data_as(C.POINTER(C.c_uint8))
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.nb_amr_mesh_create(self.ctx.h, C.byref(geom),
                                                       leaves.ctypes.data_as(C.POINTER(C.c_int32)),
                                                       leaves.shape[0], sp, C.byref(h)), "nb_amr_mesh_create")
        self.h = h
        n = self.ctx.lib.nb_amr_mesh_leaf_count(h)
        self.leaves = np.zeros((n, 4), dtype=np.int32)
        self.ctx.lib.nb_amr_mesh_leaves(h, self.leaves.ctypes.data_as(C.POINTER(C.c_int32)))

    @property
    def ncell(self) -> int:
        return self.leaves.shape[0] * 512

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.nb_amr_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def maps(self):
        """(keys, face-neighbour ranks [n,6,4], counts [n,6]) of the mesh's own tree."""
        n = self.leaves.shape[0]
        keys, _, nbr, cnt = _map_arrays(n)
        I32 = C.POINTER(C.c_int32)
        self.ctx.check(self.ctx.lib.nb_amr_mesh_maps(self.h, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                     nbr.ctypes.data_as(I32), cnt.ctypes.data_as(I32)),
                       "nb_amr_mesh_maps")
        return keys, nbr, cnt

    def couplings(self):
        """Coarse-fine couplings of the composite operator: (off [cells+1], nbr, coef)."""
        cnt = C.c_int64()
        lib = self.ctx.lib
        self.ctx.check(lib.nb_amr_mesh_couplings(self.h, C.byref(cnt), None, None, None, 0), "couplings")
        off = np.zeros(self.ncell + 1, dtype=np.int32)
        nbr = np.zeros(max(cnt.value, 1), dtype=np.int32)
        coef = np.zeros(max(cnt.value, 1))
        I32 = C.POINTER(C.c_int32)
        self.ctx.check(lib.nb_amr_mesh_couplings(self.h, C.byref(cnt), off.ctypes.data_as(I32),
                                                 nbr.ctypes.data_as(I32), abi.dptr(coef), nbr.size),
                       "couplings")
        return off, nbr[:cnt.value], coef[:cnt.value]

    def cell_size(self):
        """Per-cell (hx, hy, hz) arrays."""
        lev = np.repeat(self.leaves[:, 0], 512)
        return tuple(self.geom.h0[a] / (2.0 ** lev) for a in range(3))

    def cell_centers(self):
        lev, i, j, k = cell_coords(self.leaves)
        hx, hy, hz = self.cell_size()
        o = self.geom.origin
        return o[0] + (i + 0.5) * hx, o[1] + (j + 0.5) * hy, o[2] + (k + 0.5) * hz

    def apply_a(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(self.ncell)
        self.ctx.check(self.ctx.lib.nb_amr_apply_laplacian(self.ctx.h, self.h, abi.dptr(x), abi.dptr(out)),
                       "nb_amr_apply_laplacian")
        return out

    def solve(self, b: np.ndarray, tol=1e-10, max_cycles=200, precision=abi.PRECISION_FP64):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.ncell)
        rep = abi.PoissonReport()
        self.ctx.check(self.ctx.lib.nb_amr_poisson_solve(self.ctx.h, self.h, abi.dptr(b), abi.dptr(x), tol,
                                                         max_cycles, precision, C.byref(rep)),
                       "nb_amr_poisson_solve")
        return x, Report(rep.iterations, rep.residual, bool(rep.converged))


class AmrCase:
    """NSSolver-style MAC step on an AMR mesh, state resident on the device
    (nb_amr_case_*). Face arrays are in the library's storage order (see
    ``face_positions``)."""

    def __init__(self, mesh: AmrMesh, config: abi.FlowConfig, precision: int = abi.PRECISION_FP64):
        self.mesh, self.ctx, self.config, self.precision = mesh, mesh.ctx, config, precision
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.nb_amr_case_create(self.ctx.h, mesh.h, C.byref(config), precision,
                                                       C.byref(h)), "nb_amr_case_create")
        self.h = h
        sz = (C.c_int64 * 4)()
        self.ctx.check(self.ctx.lib.nb_amr_case_sizes(h, sz), "nb_amr_case_sizes")
        self.sizes = tuple(int(s) for s in sz)
        ncell = mesh.leaves.shape[0] * 512
        self.slabs = []
        for a in range(3):
            arr = np.zeros((self.sizes[a] - ncell) // 64, dtype=np.int32)
            if arr.size:
                self.ctx.check(self.ctx.lib.nb_amr_case_slabs(h, a, arr.ctypes.data_as(C.POINTER(C.c_int32))),
                               "nb_amr_case_slabs")
            self.slabs.append(arr)

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.nb_case_destroy(self.h)
            self.h = None

    def sample(self, component: int, points) -> np.ndarray:
        """SolverBackend::sample for many points: component 0-2 = cell-centred
        velocity of the containing cell, 3 = its pressure (nb_case_sample)."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(pts.shape[0])
        self.ctx.check(self.ctx.lib.nb_case_sample(self.h, component, pts.shape[0], abi.dptr(pts), abi.dptr(out)),
                       "nb_case_sample")
        return out

    def refine_leaves(self, sensor: int, above: float) -> np.ndarray:
        """The mesh's leaves refined on the device where sensor `sensor` exceeds
        `above` (nb_amr_case_refine: sensors, split, balance and ranking on the
        GPU); rank order."""
        n = self.mesh.leaves.shape[0]
        need = C.c_int64()
        cap = 8 * n
        out = np.zeros((cap, 4), dtype=np.int32)
        self.ctx.check(self.ctx.lib.nb_amr_case_refine(self.h, sensor, above,
                                                       out.ctypes.data_as(C.POINTER(C.c_int32)), cap,
                                                       C.byref(need)), "nb_amr_case_refine")
        return out[:need.value].copy()

    def sensors(self) -> np.ndarray:
        """Per-leaf max |vorticity|, strain magnitude, Q, |grad p| (nb_amr_case_sensors), shape (nleaf, 4)."""
        out = np.zeros((self.mesh.leaves.shape[0], 4))
        self.ctx.check(self.ctx.lib.nb_amr_case_sensors(self.h, abi.dptr(out)), "nb_amr_case_sensors")
        return out

    def transfer_from(self, src: "AmrCase"):
        """Take src's state and clock across a regrid (nb_amr_case_transfer)."""
        self.ctx.check(self.ctx.lib.nb_amr_case_transfer(self.h, src.h), "nb_amr_case_transfer")

    def write_vtu(self, path):
        """VTK XML unstructured grid of the cell-centred state (nb_case_write_vtu)."""
        self.ctx.check(self.ctx.lib.nb_case_write_vtu(self.h, str(path).encode()), "write_vtu")

    def write_checkpoint(self, path):
        """Octree checkpoint (NBFAMR1): leaf list, step clock, u, v, w, p."""
        self.ctx.check(self.ctx.lib.nb_case_write_checkpoint(self.h, str(path).encode()), "write_checkpoint")

    def read_checkpoint(self, path):
        """Restores state and step clock from an NBFAMR1 file of the same mesh."""
        self.ctx.check(self.ctx.lib.nb_case_read_checkpoint(self.h, str(path).encode()), "read_checkpoint")

    def __del__(self):
        self.close()

    def face_index(self, a: int):
        """(level, i, j, k) face coordinates of every stored a-face, storage
        order: i, j, k are level-`level` indices with the a-th one the face
        index (low face of cell i is i; a slab face is 8*b + 8)."""
        lv = self.mesh.leaves
        lev, i, j, k = cell_coords(lv)
        idx = [i, j, k]
        sl = self.slabs[a]
        if sl.size:
            m = np.arange(64)
            t1, t2 = [(1, 2), (0, 2), (0, 1)][a]
            sb = lv[sl]
            slev = np.repeat(sb[:, 0], 64)
            sidx = [None, None, None]
            sidx[a] = np.repeat(sb[:, 1 + a] * 8 + 8, 64)
            sidx[t1] = (sb[:, 1 + t1:2 + t1] * 8 + (m & 7)[None, :]).ravel()
            sidx[t2] = (sb[:, 1 + t2:2 + t2] * 8 + (m >> 3)[None, :]).ravel()
            lev = np.concatenate([lev, slev])
            idx = [np.concatenate([idx[d], sidx[d]]) for d in range(3)]
        return lev, idx[0], idx[1], idx[2]

    def face_positions(self, a: int):
        """Physical (x, y, z) of every stored a-face (storage order)."""
        lev, i, j, k = self.face_index(a)
        h = [self.mesh.geom.h0[d] / (2.0 ** lev) for d in range(3)]
        o = self.mesh.geom.origin
        idx = (i, j, k)
        return [o[d] + (idx[d] + (0.0 if d == a else 0.5)) * h[d] for d in range(3)]

    def initialize(self):
        self.ctx.check(self.ctx.lib.nb_case_initialize(self.h), "initialize")

    def set_state(self, u, v, w, p):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, w, p)]
        if [x.size for x in arrs] != list(self.sizes):
            raise ValueError(f"state sizes {[x.size for x in arrs]} != {list(self.sizes)}")
        self.ctx.check(self.ctx.lib.nb_amr_case_set_state(self.h, *[abi.dptr(x) for x in arrs]), "set_state")

    def get_state(self, out=None):
        """Face velocities and pressure in the case's layout. `out`: four
        contiguous float64 arrays of the right sizes to copy into (pinned
        buffers make the read-back one DMA per array, no host copy)."""
        if out is None:
            out = [np.zeros(n) for n in self.sizes]
        elif [x.size for x in out] != list(self.sizes) or not all(
                x.dtype == np.float64 and x.flags.c_contiguous and x.flags.writeable for x in out):
            raise ValueError("get_state: out must be four writeable contiguous float64 arrays of the state sizes")
        self.ctx.check(self.ctx.lib.nb_amr_case_get_state(self.h, *[abi.dptr(x) for x in out]), "get_state")
        return out

    def compute_dt(self) -> float:
        dt = C.c_double()
        self.ctx.check(self.ctx.lib.nb_case_compute_dt(self.h, C.byref(dt)), "computeDt")
        return dt.value

    def step(self, dt: float = 0.0) -> abi.StepReport:
        rep = abi.StepReport()
        self.ctx.check(self.ctx.lib.nb_step(self.h, dt, C.byref(rep)), "step")
        return rep

    def step_many(self, dt: float, n: int) -> abi.StepReport:
        rep = abi.StepReport()
        self.ctx.check(self.ctx.lib.nb_step_many(self.h, dt, n, C.byref(rep)), "step_many")
        return rep

    @property
    def cell_count(self) -> int:
        return self.ctx.lib.nb_case_cell_count(self.h)


def regrid(case: AmrCase, refine_above: float, coarsen_below: float, sensor: int = 0, solid_fn=None,
           device: bool = True) -> AmrCase:
    """One regrid pass on the device sensors: leaves whose sensor `sensor`
    (0 |vorticity|, 1 strain, 2 Q, 3 |grad p|) exceeds refine_above are split
    (2:1 balance restored; on the device by default, nb_amr_case_refine, else
    by the host maps), then complete octets of untouched leaves below
    coarsen_below are merged; a new case on the new mesh takes the state
    conservatively. solid_fn(leaves) -> per-cell solid flags (leaves x 512, in
    leaf order) or None. Returns the new case (the old one is left as it was)."""
    mesh = case.mesh
    geom, leaves = mesh.geom, mesh.leaves
    s = case.sensors()[:, sensor]
    if device:
        refined = case.refine_leaves(sensor, refine_above)
    else:
        refined = refine(geom, leaves, (s > refine_above) & (leaves[:, 0] < geom.lmax))
    # leaves the refinement left alone keep their sensor value; new ones are not coarsened
    old = {tuple(l): v for l, v in zip(map(tuple, leaves), s)}
    flags = np.array([old.get(tuple(l), np.inf) < coarsen_below for l in refined], dtype=np.uint8)
    new_leaves = coarsen(geom, refined, flags)
    solid = solid_fn(new_leaves) if solid_fn else None
    new_mesh = AmrMesh(geom, new_leaves, solid=solid, ctx=case.ctx)
    new = AmrCase(new_mesh, case.config, precision=case.precision)
    new.transfer_from(case)
    new._mesh_keepalive = new_mesh
    return new
