"""Shared test helpers: grids of the reference's own tests and comparisons."""
import numpy as np

from nabla_b200 import abi, cases


def rel_err(a, b):
    """max |a - b| / max |b| (0/0 -> 0)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if a.size else 0.0
    return 0.0 if num == 0.0 else num / max(den, 1e-300)


def channel_block_grid():
    """Operator of core/tests/test_flow.cpp:63-86: 32x16x16, inlet/outlet/walls/
    periodic span, wall-mounted solid block."""
    faces = [dict(type=abi.BC_INLET), dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL),
             dict(type=abi.BC_WALL), dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = cases.Grid(32, 16, 16, 1 / 16, 1 / 16, 1 / 16, faces=faces)
    s = g.solid.reshape(16, 16, 32)
    s[6:10, 0:6, 12:18] = 1
    return g


def periodic2d_grid(n):
    """core/tests/test_flow.cpp:21-30 / :119-129: n x n x 1, all periodic, h = 1/n."""
    return cases.Grid(n, n, 1, 1.0 / n, 1.0 / n, 1.0 / n, faces=cases.periodic_faces())


def mixed_bc_grid(nx=12, ny=10, nz=9, seed=3):
    """Partial bricks (sizes not multiples of 8), every BC kind and random solids."""
    faces = [dict(type=abi.BC_INLET, profile=abi.PROFILE_PARABOLIC, inlet_speed=1.3, inlet_axis=0),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL, wall_velocity=(0.2, 0.0, 0.1)),
             dict(type=abi.BC_WALL), dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC)]
    g = cases.Grid(nx, ny, nz, 0.11, 0.09, 0.1, origin=(0.3, -0.2, 0.1), faces=faces)
    rng = np.random.default_rng(seed)
    g.solid[:] = (rng.random(g.ncell) < 0.08).astype(np.uint8)
    return g


def closed_box_grid(n=16, seed=5):
    """All-wall closed box with solids (singular, non-periodic)."""
    g = cases.Grid(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, faces=[dict(type=abi.BC_WALL) for _ in range(6)])
    rng = np.random.default_rng(seed)
    g.solid[:] = (rng.random(g.ncell) < 0.05).astype(np.uint8)
    return g
