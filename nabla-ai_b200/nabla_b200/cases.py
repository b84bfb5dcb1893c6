"""Case builders: grids, boundary conditions and seeded initial states.

Mirrors the reference's case builders (core/src/flow/case.cpp:25-134:
makeLidCavity, makeChannel, makeWallMountedCube) and adds the synthetic
workloads the benchmarks run (Taylor-Green vortex on the periodic box,
the obstacle channel). Everything here is host-side set-up; the solver
path itself is the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class Grid:
    """Owns a GridDesc plus the numpy solid mask it points to."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    origin: tuple = (0.0, 0.0, 0.0)
    faces: list = field(default_factory=lambda: [dict(type=abi.BC_WALL) for _ in range(6)])
    solid: np.ndarray | None = None

    def __post_init__(self):
        if self.solid is None:
            self.solid = np.zeros(self.nx * self.ny * self.nz, dtype=np.uint8)
        self.solid = np.ascontiguousarray(self.solid, dtype=np.uint8).reshape(-1)
        assert self.solid.size == self.nx * self.ny * self.nz

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def sizes(self):
        """(len u, len v, len w, len p) in the staggered lexicographic layout."""
        nx, ny, nz = self.nx, self.ny, self.nz
        return (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1), nx * ny * nz

    def desc(self) -> abi.GridDesc:
        d = abi.GridDesc()
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.origin[:] = list(self.origin)
        d.dx, d.dy, d.dz = self.dx, self.dy, self.dz
        for f in range(6):
            spec = self.faces[f]
            d.face[f].type = spec.get("type", abi.BC_WALL)
            d.face[f].profile = spec.get("profile", abi.PROFILE_UNIFORM)
            d.face[f].inlet_axis = spec.get("inlet_axis", 0)
            d.face[f].inlet_speed = spec.get("inlet_speed", 0.0)
            wv = spec.get("wall_velocity", (0.0, 0.0, 0.0))
            d.face[f].wall_velocity[:] = list(wv)
        d.solid = self.solid.ctypes.data_as(C.POINTER(C.c_uint8))
        self._keep = d  # keep alive alongside the numpy buffer
        return d

    def cell_center(self, i, j, k):
        return (self.origin[0] + (i + 0.5) * self.dx, self.origin[1] + (j + 0.5) * self.dy,
                self.origin[2] + (k + 0.5) * self.dz)


def flow_config(reynolds=100.0, ref_length=1.0, velocity_scale=1.0, density=1.0, cfl=0.8,
                body_force=(0.0, 0.0, 0.0), convection=abi.CONV_CENTRAL, poisson_tol=1e-9,
                poisson_max_iters=5000, tol_continuity=1e-7, tol_mass=1e-8,
                ref_area=0.0) -> abi.FlowConfig:
    """FlowConfig with the reference defaults (core/include/nabla/flow/ns_solver.hpp:14-32)."""
    c = abi.FlowConfig()
    c.reynolds, c.ref_length, c.velocity_scale = reynolds, ref_length, velocity_scale
    c.density, c.cfl = density, cfl
    c.body_force[:] = list(body_force)
    c.convection, c.poisson_max_iters, c.poisson_tol = convection, poisson_max_iters, poisson_tol
    c.tol_continuity, c.tol_mass, c.ref_area = tol_continuity, tol_mass, ref_area
    return c


def periodic_faces():
    return [dict(type=abi.BC_PERIODIC) for _ in range(6)]


# ---- reference builders (core/src/flow/case.cpp:25-134) -------------------
def lid_cavity(n, reynolds, lid_velocity=1.0):
    faces = [dict(type=abi.BC_WALL) for _ in range(6)]
    faces[4] = dict(type=abi.BC_PERIODIC)
    faces[5] = dict(type=abi.BC_PERIODIC)
    faces[3] = dict(type=abi.BC_WALL, wall_velocity=(lid_velocity, 0.0, 0.0))
    g = Grid(n, n, 1, 1.0 / n, 1.0 / n, 1.0 / n, faces=faces)
    cfg = flow_config(reynolds=reynolds, velocity_scale=lid_velocity, cfl=0.8)
    return g, cfg


def channel(nx, ny, reynolds, bulk=1.0):
    Ly, Lx = 1.0, 6.0
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_PARABOLIC, inlet_speed=bulk, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = Grid(nx, ny, 1, Lx / nx, Ly / ny, Ly / ny, faces=faces)
    cfg = flow_config(reynolds=reynolds, ref_length=Ly, velocity_scale=bulk, cfl=0.8)
    return g, cfg


def wall_mounted_cube(resolution, reynolds):
    h = 1.0
    nx, ny, nz = round(14.0 * resolution), round(3.0 * resolution), round(6.4 * resolution)
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_UNIFORM, inlet_speed=1.0, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL),
             dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = Grid(nx, ny, nz, h / resolution, h / resolution, h / resolution, faces=faces)
    x0, x1, y0, y1 = 3.0 * h, 4.0 * h, 0.0, h
    zc = 3.2 * h
    z0, z1 = zc - 0.5 * h, zc + 0.5 * h
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cx, cy, cz = (i + 0.5) * g.dx, (j + 0.5) * g.dy, (k + 0.5) * g.dz
    inside = (cx >= x0) & (cx <= x1) & (cy >= y0) & (cy <= y1) & (cz >= z0) & (cz <= z1)
    g.solid[:] = inside.reshape(-1).astype(np.uint8)
    cfg = flow_config(reynolds=reynolds, ref_length=h, velocity_scale=1.0, ref_area=h * h, cfl=0.7,
                      convection=abi.CONV_WENO5)
    return g, cfg


# ---- Taylor-Green vortex on the periodic box [0, 2pi]^3 --------------------
def taylor_green(n=64, reynolds=1600.0, cfl=0.4, poisson_tol=1e-10):
    """Periodic TGV box: n^3 cells of 2pi/n, nu = 1/reynolds, WENO-5."""
    L = 2.0 * math.pi
    g = Grid(n, n, n, L / n, L / n, L / n, faces=periodic_faces())
    cfg = flow_config(reynolds=reynolds, ref_length=1.0, velocity_scale=1.0, cfl=cfl,
                      convection=abi.CONV_WENO5, poisson_tol=poisson_tol)
    return g, cfg


def taylor_green_state(g: Grid):
    """Analytic TGV on the MAC faces: u = sin x cos y cos z at x-faces,
    v = -cos x sin y cos z at y-faces, w = 0, p from the analytic solution
    p = (cos 2x + cos 2y)(cos 2z + 2)/16 at cell centres."""
    nx, ny, nz = g.nx, g.ny, g.nz
    dx, dy, dz = g.dx, g.dy, g.dz
    ox, oy, oz = g.origin
    xf = ox + np.arange(nx + 1) * dx
    xc = ox + (np.arange(nx) + 0.5) * dx
    yf = oy + np.arange(ny + 1) * dy
    yc = oy + (np.arange(ny) + 0.5) * dy
    zc = oz + (np.arange(nz) + 0.5) * dz
    u = (np.sin(xf)[None, None, :] * np.cos(yc)[None, :, None] * np.cos(zc)[:, None, None])
    v = (-np.cos(xc)[None, None, :] * np.sin(yf)[None, :, None] * np.cos(zc)[:, None, None])
    w = np.zeros((nz + 1, ny, nx))
    p = ((np.cos(2 * xc)[None, None, :] + np.cos(2 * yc)[None, :, None]) *
         (np.cos(2 * zc)[:, None, None] + 2.0) / 16.0)
    return (np.ascontiguousarray(u.reshape(-1)), np.ascontiguousarray(v.reshape(-1)),
            np.ascontiguousarray(w.reshape(-1)), np.ascontiguousarray(p.reshape(-1)))


def random_state(g: Grid, seed: int, amp: float = 1.0):
    """Seeded uniform(-amp, amp) staggered state (parity tests)."""
    rng = np.random.default_rng(seed)
    nu, nv, nw, np_ = g.sizes()
    return (rng.uniform(-amp, amp, nu), rng.uniform(-amp, amp, nv), rng.uniform(-amp, amp, nw),
            rng.uniform(-amp, amp, np_))
