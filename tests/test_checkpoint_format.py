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


def _case_files(tmp_path):
    import json
    specs = {
        "cavity.json": {"type": "lid-cavity", "name": "c", "reynolds": 100, "resolution": 24, "cfl": 0.8,
                        "convection": "central", "max_steps": 80, "steady_tol": 1e-5, "run_dir": "rc"},
        "channel.json": {"type": "channel", "reynolds": 50, "resolution": 8, "nx": 40, "bulk_velocity": 1.5,
                         "checkpoint_every": 7},
        "cube.json": {"type": "wall-mounted-cube", "reynolds": 300, "resolution": 4, "convection": "weno5",
                      "stop_time": 2.5, "precision": "mixed"},
    }
    out = []
    for name, spec in specs.items():
        p = tmp_path / name
        p.write_text(json.dumps(spec))
        out.append(p)
    return out


def test_load_case_matches_the_reference(ref, tmp_path):
    """solver.load_case against the reference's own loadCase on the same files."""
    for path in _case_files(tmp_path):
        g, solid, cfg, run = ref.load_case(path)
        spec = solver.load_case(path)
        d = spec["grid"].desc()
        for f in ("nx", "ny", "nz", "dx", "dy", "dz"):
            assert getattr(d, f) == getattr(g, f), (path.name, f)
        assert tuple(d.origin) == tuple(g.origin)
        for q in range(6):
            for f in ("type", "profile", "inlet_axis", "inlet_speed"):
                assert getattr(d.face[q], f) == getattr(g.face[q], f), (path.name, q, f)
            assert tuple(d.face[q].wall_velocity) == tuple(g.face[q].wall_velocity)
        assert np.array_equal(np.asarray(spec["grid"].solid, dtype=np.uint8), solid)
        c = spec["config"]
        for f, _ in cfg._fields_:
            a, b = getattr(c, f), getattr(cfg, f)
            assert (tuple(a) == tuple(b)) if f == "body_force" else a == b, (path.name, f)
        r = dict(spec["run"])
        r.pop("restart_from")
        assert r == run, path.name
    assert solver.load_case(_case_files(tmp_path)[2])["precision"] == 1
