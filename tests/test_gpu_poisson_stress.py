"""Pressure-solve precision stress on a 3-level octree (effective 128^3 TGV
box): a seeded N(0,1) right-hand side projected to zero volume-weighted mean,
solved to 1e-12 relative residual by FP64 MG-PCG and by the mixed form (FP32
V-cycle inside the FP64 flexible PCG, FP64 true residual). Both must converge;
the mixed pressure must agree with the FP64 one to 1e-9 relative (max norm)
and its discrete divergence residual must meet the tolerance."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, workloads

pytestmark = pytest.mark.gpu


def test_mixed_solve_matches_fp64_at_1e_12(ctx):
    geom, leaves = workloads.tgv_octree(32)
    assert leaves[:, 0].max() == 2
    mesh = amr.AmrMesh(geom, leaves, ctx=ctx)
    b = np.random.default_rng(32).standard_normal(mesh.ncell)
    hx, hy, hz = mesh.cell_size()
    vol = hx * hy * hz
    b -= np.sum(vol * b) / vol.sum()
    x64, r64 = mesh.solve(b, 1e-12, 400, precision=abi.PRECISION_FP64)
    x32, r32 = mesh.solve(b, 1e-12, 400, precision=abi.PRECISION_MIXED)
    assert r64.converged and r32.converged
    assert r32.iterations <= 2 * r64.iterations + 2
    assert np.abs(x32 - x64).max() / np.abs(x64).max() < 1e-9
    res = mesh.apply_a(x32) - b
    assert np.sqrt(np.sum(vol * res * res) / np.sum(vol * b * b)) < 1e-11
