"""Generate the golden fixtures from the reference's own CPU code.

    make -C oracle REF=<reference checkout> ref && python tests/golden/make_golden.py

Runs the reference (oracle/_ref/libnabla_ref.so, compiled in place from the
reference tree by oracle/Makefile) on small seeded inputs and stores inputs
and outputs in tests/golden/*.npz. The fixtures pin the oracle restatement and
the CUDA path without the reference tree being present.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "nabla-ai_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "tests"))

import oracle  # noqa: E402
from helpers import channel_block_grid, closed_box_grid, mixed_bc_grid, periodic2d_grid  # noqa: E402
from nabla_b200 import abi, cases  # noqa: E402


def rep_dict(r):
    return {k: np.float64(v) for k, v in r.as_dict().items()}


def main():
    R = oracle.Reference()
    out = {}
    # 1. -Laplacian on partial bricks with every BC kind (poisson.cpp:102-134)
    g = mixed_bc_grid()
    x = np.random.default_rng(11).uniform(-1, 1, g.ncell)
    out["applyA_mixed_x"] = x
    out["applyA_mixed_Ax"] = R.apply_a(g, x)
    out["applyA_mixed_solid"] = g.solid.copy()
    # 2. MG-PCG on the reference test operator (core/tests/test_flow.cpp:63-117):
    #    x_exact ~ U(-1,1) from mt19937(12345) on fluid cells, b = A x_exact.
    g = channel_block_grid()
    fluid = np.flatnonzero(g.solid == 0)
    xe = np.zeros(g.ncell)
    xe[fluid] = R.uniform(12345, fluid.size)
    b = R.apply_a(g, xe)
    x, rep = R.poisson(g, b, 1e-10, 100)
    out["mg_channel_b"] = b
    out["mg_channel_xexact"] = xe
    out["mg_channel_x"] = x
    out["mg_channel_rep"] = np.array([rep.iterations, rep.residual, rep.converged], dtype=np.float64)
    # 3. MG-PCG, singular periodic 24x24 (core/tests/test_flow.cpp:119-159)
    g = periodic2d_grid(24)
    i, j = np.meshgrid(np.arange(24), np.arange(24), indexing="xy")
    phi = (np.cos(2 * np.pi * (i + 0.5) / 24) * np.cos(2 * np.pi * (j + 0.5) / 24)).reshape(-1)
    b = R.apply_a(g, phi)
    x, rep = R.poisson(g, b, 1e-12, 100)
    out["mg_periodic_b"] = b
    out["mg_periodic_x"] = x
    out["mg_periodic_rep"] = np.array([rep.iterations, rep.residual, rep.converged], dtype=np.float64)
    # 4. closed box with solids, singular non-periodic
    g = closed_box_grid()
    b = np.random.default_rng(21).standard_normal(g.ncell)
    x, rep = R.poisson(g, b, 1e-10, 100)
    out["mg_box_solid"] = g.solid.copy()
    out["mg_box_b"] = b
    out["mg_box_x"] = x
    out["mg_box_rep"] = np.array([rep.iterations, rep.residual, rep.converged], dtype=np.float64)
    # 5. Taylor-Green 16^3, WENO-5, dt = computeDt at CFL 0.4, 2 steps
    g, cfg = cases.taylor_green(16)
    st = cases.taylor_green_state(g)
    ns = R.ns(g, cfg)
    ns.set_state(*st)
    dt = ns.compute_dt()
    out["tgv16_dt"] = np.float64(dt)
    for s in range(2):
        r = ns.step(dt)
        u, v, w, p = ns.get_state()
        out[f"tgv16_s{s + 1}_u"], out[f"tgv16_s{s + 1}_v"] = u, v
        out[f"tgv16_s{s + 1}_w"], out[f"tgv16_s{s + 1}_p"] = w, p
        out[f"tgv16_s{s + 1}_rep"] = np.array([r.poisson_iters, r.continuity_residual,
                                               r.divergence_max, r.momentum_residual])
    # 6. wall-mounted cube, resolution 2 (28x6x13), WENO-5, CFL dt, 2 steps
    g, cfg = cases.wall_mounted_cube(2, 200.0)
    ns = R.ns(g, cfg)
    ns.initialize()
    for s in range(2):
        r = ns.step()
        u, v, w, p = ns.get_state()
        out[f"cube2_s{s + 1}_u"], out[f"cube2_s{s + 1}_v"] = u, v
        out[f"cube2_s{s + 1}_w"], out[f"cube2_s{s + 1}_p"] = w, p
        out[f"cube2_s{s + 1}_rep"] = np.array([r.dt, r.poisson_iters, r.cd, r.cl, r.mass_error])
    # 7. Morton keys (core/tests/test_morton.cpp:10-39): coords from mt19937_64(0xC0FFEE)
    coords = (R.uniform(0xC0FFEE, 3 * 200, 0.0, 2097151.0, bits64=True)).astype(np.uint32).reshape(-1, 3)
    out["morton_coords"] = coords
    out["morton_keys"] = np.array([R.morton_encode(int(a), int(b_), int(c)) for a, b_, c in coords],
                                  dtype=np.uint64)
    path = os.path.join(HERE, "reference_small.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
