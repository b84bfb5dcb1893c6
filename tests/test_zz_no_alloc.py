"""The allocation-free -Laplacian entry point (nb_apply_laplacian_noalloc).

It serves callers that cannot call cudaMalloc (hosts that own all device
memory through their own arena or admission budget). The test allocates the
caller's device buffers with torch, calls the entry point through the C ABI
three times in a row with different grids (the second one without a solid
mask, so the shared static scratch must be fully rewritten; the third a 2-D
grid, nz = 1, which skips the z coupling as the reference's 2-D case does),
and checks each result against the allocating entry point nb_apply_laplacian
at the operator tolerance used elsewhere (1e-13 relative).

This file is collected last so a failure here cannot hide other results.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import channel_block_grid, mixed_bc_grid, rel_err
from nabla_b200 import abi, solver

pytestmark = pytest.mark.gpu


def _noalloc(lib, desc, x_np):
    import torch
    xd = torch.from_numpy(x_np).cuda()
    od = torch.full_like(xd, float("nan"))
    stream = torch.cuda.current_stream()
    st = lib.nb_apply_laplacian_noalloc(C.byref(desc), C.c_void_p(xd.data_ptr()),
                                        C.c_void_p(od.data_ptr()), C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return st, od.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_in_a_row():
    ctx = solver.default_context()
    lib = abi.load()
    # call 1: partial bricks, every BC kind, random solids
    g1 = mixed_bc_grid(21, 11, 13, seed=17)
    x1 = np.random.default_rng(31).uniform(-1, 1, g1.ncell)
    st, got1 = _noalloc(lib, g1.desc(), x1)
    assert st == abi.NB_OK
    assert rel_err(got1, solver.apply_a(g1, x1, ctx)) < 1e-13
    # call 2: different grid, NULL solid mask (the scratch must not keep call 1's mask)
    g2 = channel_block_grid()
    g2.solid[:] = 0
    d2 = g2.desc()
    d2.solid = C.POINTER(C.c_uint8)()
    x2 = np.random.default_rng(32).uniform(-1, 1, g2.ncell)
    st, got2 = _noalloc(lib, d2, x2)
    assert st == abi.NB_OK
    assert rel_err(got2, solver.apply_a(g2, x2, ctx)) < 1e-13
    # call 3: 2-D grid (nz = 1), periodic x, inlet / outlet in y, solids
    from nabla_b200 import cases
    faces = [dict(type=abi.BC_PERIODIC), dict(type=abi.BC_PERIODIC), dict(type=abi.BC_INLET),
             dict(type=abi.BC_OUTLET), dict(type=abi.BC_WALL), dict(type=abi.BC_WALL)]
    g3 = cases.Grid(19, 14, 1, 0.07, 0.05, 0.05, faces=faces)
    g3.solid[:] = (np.random.default_rng(33).random(g3.ncell) < 0.1).astype(np.uint8)
    x3 = np.random.default_rng(34).uniform(-1, 1, g3.ncell)
    st, got3 = _noalloc(lib, g3.desc(), x3)
    assert st == abi.NB_OK
    assert rel_err(got3, solver.apply_a(g3, x3, ctx)) < 1e-13


def test_noalloc_rejects_oversize_grid():
    lib = abi.load()
    from nabla_b200 import cases
    g = cases.Grid(1, 1, 1, 1.0, 1.0, 1.0)
    d = g.desc()
    d.nx, d.ny, d.nz = 512, 512, 128  # 2^25 cells > NB_NOALLOC_MAX_CELLS
    st = lib.nb_apply_laplacian_noalloc(C.byref(d), C.c_void_p(8), C.c_void_p(8), None)
    assert st == abi.NB_ERR_UNSUPPORTED
