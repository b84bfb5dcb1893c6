"""The case run loop (nb_run_case) against the reference's runCase
(core/src/flow/case.cpp:349-401) on the same channel: diagnostics.jsonl
records with the same keys in the same order and matching values, the same
checkpoint files with states within 1e-10 relative, the same final.vtu
(writeGridVtu, case.cpp:175-241) to its 8 printed digits, and a restart from
an intermediate checkpoint that ends bit for bit on the uninterrupted run.
Octree cases write every leaf cell with its level."""
import json
import struct

import numpy as np
import pytest

from nabla_b200 import cases, solver

pytestmark = pytest.mark.gpu

PHYSICAL = ("t", "dt", "cfl", "momentum_residual", "cd", "cl")
RESIDUAL = ("continuity_residual", "divergence_max", "mass_error", "poisson_residual")


def _records(path):
    return [json.loads(line) for line in open(path).read().splitlines()]


def _ckpt(path):
    raw = open(path, "rb").read()
    assert raw[:8] == b"NBFCK01\0"
    off, arrs = 40, []
    for _ in range(4):
        (n,) = struct.unpack_from("<Q", raw, off)
        arrs.append(np.frombuffer(raw, dtype="<f8", count=n, offset=off + 8))
        off += 8 + 8 * n
    return struct.unpack_from("<i", raw, 20)[0], arrs


def _vtu(path):
    """Points, the three cell arrays and every CellData array of a VTU file."""
    import xml.etree.ElementTree as ET
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {}
    for da in piece.iter("DataArray"):
        arrays[da.get("Name") or "points"] = np.array(da.text.split(), dtype=np.float64)
    return int(piece.get("NumberOfCells")), arrays


def _channel():
    grid, cfg = cases.channel(32, 16, 100.0, 1.0)
    cfg.poisson_tol = 1e-9
    return grid, cfg


def test_run_case_matches_reference(ctx, ref, tmp_path):
    grid, cfg = _channel()
    rd, gd = tmp_path / "ref", tmp_path / "gpu"
    rs = ref.run_case(grid, cfg, rd, 12, checkpoint_every=5)
    gs = solver.run_case(grid, cfg, gd, 12, checkpoint_every=5, ctx=ctx)
    assert gs["steps"] == rs["steps"] == 12 and not gs["steady"]
    assert gs["time"] == pytest.approx(rs["time"], rel=1e-10)
    R, G = _records(rd / "diagnostics.jsonl"), _records(gd / "diagnostics.jsonl")
    assert len(R) == len(G) == 13
    assert R[0]["event"] == G[0]["event"] == "meta" and list(R[0]) == list(G[0])
    assert G[0]["solver"] == "nabla_b200"
    for r, g in zip(R[1:], G[1:]):
        assert list(g) == list(r)
        for k in ("step", "poisson_iters", "cells", "accepted"):
            assert g[k] == r[k], k
        for k in PHYSICAL:  # printed with 6 significant digits
            assert g[k] == pytest.approx(r[k], rel=2e-5, abs=1e-12), k
        for k in RESIDUAL:  # solver-tolerance quantities: same order of magnitude
            assert abs(g[k]) <= max(10 * abs(r[k]), 1e-9), k
    nr, ra = _vtu(rd / "final.vtu")
    ng, ga = _vtu(gd / "final.vtu")
    assert ng == nr == grid.nx * grid.ny * grid.nz and set(ga) == set(ra)
    for k in ("points", "connectivity", "offsets", "types", "solid"):
        assert np.array_equal(ga[k], ra[k]), k
    for k in ("u", "v", "w", "p", "speed"):  # 8 significant digits in the file
        assert np.allclose(ga[k], ra[k], rtol=1e-6, atol=1e-9 * np.abs(ra[k]).max()), k
    for name in ("checkpoint_5.ckpt", "checkpoint_10.ckpt", "final.ckpt"):
        rstep, ra = _ckpt(rd / name)
        gstep, ga = _ckpt(gd / name)
        assert gstep == rstep
        for x, y in zip(ga, ra):
            assert np.abs(x - y).max() <= 1e-10 * max(np.abs(y).max(), 1e-30)


def test_run_case_restart_is_bit_exact(ctx, tmp_path):
    grid, cfg = _channel()
    full, part = tmp_path / "full", tmp_path / "part"
    solver.run_case(grid, cfg, full, 12, checkpoint_every=5, ctx=ctx)
    s = solver.run_case(grid, cfg, part, 7, restart_from=full / "checkpoint_5.ckpt", ctx=ctx)
    assert s["steps"] == 12
    steps = [r["step"] for r in _records(part / "diagnostics.jsonl")]
    assert steps == list(range(6, 13))  # a restart appends step records only
    _, a = _ckpt(full / "final.ckpt")
    _, b = _ckpt(part / "final.ckpt")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    with pytest.raises(solver.NablaError, match="cannot open"):
        solver.run_case(grid, cfg, tmp_path / "bad", 1, restart_from=tmp_path / "missing.ckpt", ctx=ctx)


def test_octree_vtu(ctx, tmp_path):
    from amr_helpers import closed_box_geom, two_level_leaves
    from nabla_b200 import abi, amr
    geom = closed_box_geom()
    mesh = amr.AmrMesh(geom, two_level_leaves(geom), ctx=ctx)
    ac = amr.AmrCase(mesh, cases.flow_config(reynolds=100.0, convection=abi.CONV_WENO5))
    rng = np.random.default_rng(7)
    ac.set_state(*[rng.uniform(-1, 1, n) for n in ac.sizes])
    ac.write_vtu(tmp_path / "o.vtu")
    n, arr = _vtu(tmp_path / "o.vtu")
    assert n == mesh.ncell and arr["points"].size == 24 * n
    assert np.array_equal(arr["level"], np.repeat(mesh.leaves[:, 0], 512))
    x, y, z = mesh.cell_centers()
    pts = np.stack([x, y, z], axis=1)
    for c, k in enumerate("uvwp"):
        want = ac.sample(c, pts)
        assert np.allclose(arr[k], want, rtol=1e-7, atol=1e-12), k
    corners = arr["points"].reshape(n, 8, 3)
    assert np.allclose(corners.mean(axis=1), pts, rtol=0, atol=1e-12)


def test_case_file_run_matches_reference(ctx, ref, tmp_path):
    """`nabla_solve run <case.json>` on the GPU (solver.run_case_file) against the
    reference's runCase on the same file's spec."""
    path = tmp_path / "cavity.json"
    gd = tmp_path / "gpu"
    path.write_text(json.dumps({"type": "lid-cavity", "reynolds": 100, "resolution": 24, "cfl": 0.8,
                                "convection": "central", "max_steps": 6, "run_dir": str(gd),
                                "checkpoint_every": 3, "backend": "cuda", "precision": "fp64"}))
    spec = solver.load_case(path)
    rd = tmp_path / "ref"
    ref.run_case(spec["grid"], spec["config"], rd, 6, checkpoint_every=3)
    s = solver.run_case_file(path, ctx=ctx)
    assert s["steps"] == 6
    R, G = _records(rd / "diagnostics.jsonl"), _records(gd / "diagnostics.jsonl")
    assert [r["poisson_iters"] for r in R[1:]] == [g["poisson_iters"] for g in G[1:]]
    for r, g in zip(R[1:], G[1:]):
        for k in PHYSICAL:
            assert g[k] == pytest.approx(r[k], rel=2e-5, abs=1e-12), k
    for name in ("checkpoint_3.ckpt", "checkpoint_6.ckpt", "final.ckpt", "final.vtu"):
        assert (gd / name).exists() and (rd / name).exists()
    with pytest.raises(ValueError, match="backend"):
        path.write_text(json.dumps({"type": "lid-cavity", "backend": "cpu"}))
        solver.load_case(path)
