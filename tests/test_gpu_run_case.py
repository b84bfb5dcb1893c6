"""The case run loop (nb_run_case) against the reference's runCase
(core/src/flow/case.cpp:349-401) on the same channel: diagnostics.jsonl
records with the same keys in the same order and matching values, the same
checkpoint files with states within 1e-10 relative, and a restart from an
intermediate checkpoint that ends bit for bit on the uninterrupted run."""
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
