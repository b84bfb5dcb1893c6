"""Checkpoint file format on the host: a file written by the compiled
reference's writeCheckpoint (core/src/flow/case.cpp:274-294) is read back by
nb_checkpoint_info and by the documented NBFCK01 layout (magic, int32 nx ny
nz, int32 step, FP64 t, FP64 dt, four uint64-counted FP64 arrays) with the
reference's own state, bit for bit. No GPU is needed."""
import struct

import numpy as np

from nabla_b200 import cases, solver


def _parse(path):
    raw = open(path, "rb").read()
    assert raw[:8] == b"NBFCK01\0"
    nx, ny, nz, step = struct.unpack_from("<4i", raw, 8)
    t, dt = struct.unpack_from("<2d", raw, 24)
    off, arrs = 40, []
    for _ in range(4):
        (n,) = struct.unpack_from("<Q", raw, off)
        off += 8
        arrs.append(np.frombuffer(raw, dtype="<f8", count=n, offset=off))
        off += 8 * n
    assert off == len(raw)
    return (nx, ny, nz), step, t, dt, arrs


def test_reference_checkpoint_layout(ref, tmp_path):
    grid, cfg = cases.channel(16, 8, 100.0)
    ns = ref.ns(grid, cfg)
    ns.initialize()
    ns.step()
    rep = ns.step()
    path = tmp_path / "ref.ckpt"
    ns.write_checkpoint(path)
    dims, step, t, dt, arrs = _parse(path)
    assert dims == (grid.nx, grid.ny, grid.nz) and step == 2
    assert t == rep.t and dt == rep.dt
    for a, b in zip(arrs, ns.get_state()):
        assert np.array_equal(a, b)
    info = solver.checkpoint_info(path)
    assert info == {"kind": "uniform", "step": 2, "t": rep.t, "dt": rep.dt, "dims": dims}


def test_checkpoint_info_rejects_foreign_files(tmp_path):
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(b"NOTACKPT" + bytes(64))
    assert solver.checkpoint_info(bad) is None
    short = tmp_path / "short.ckpt"
    short.write_bytes(b"NBFCK01\0" + bytes(6))
    assert solver.checkpoint_info(short) is None
    assert solver.checkpoint_info(tmp_path / "missing.ckpt") is None


def test_reference_run_directory(ref, tmp_path):
    """The reference's runCase output that nb_run_case reproduces: a meta line,
    one record per step with these keys in this order, checkpoint files."""
    import json
    grid, cfg = cases.channel(16, 8, 100.0)
    s = ref.run_case(grid, cfg, tmp_path, 3, checkpoint_every=2)
    assert s["steps"] == 3
    lines = [json.loads(x) for x in (tmp_path / "diagnostics.jsonl").read_text().splitlines()]
    assert list(lines[0]) == ["event", "solver", "solver_version", "git_sha"]
    assert [r["step"] for r in lines[1:]] == [1, 2, 3]
    assert list(lines[1]) == ["step", "t", "dt", "cfl", "momentum_residual", "continuity_residual",
                              "divergence_max", "mass_error", "cd", "cl", "poisson_iters", "poisson_residual",
                              "cells", "accepted"]
    assert solver.checkpoint_info(tmp_path / "checkpoint_2.ckpt")["step"] == 2
    assert solver.checkpoint_info(tmp_path / "final.ckpt")["step"] == 3
