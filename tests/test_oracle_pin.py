"""Pins the oracle restatement (oracle/restate*.c) to the reference.

Against the committed golden fixtures (generated by the reference's own CPU
code, tests/golden/make_golden.py) always; against the live reference library
(oracle/_ref) when it is present. CPU only.
"""
import os

import numpy as np
import pytest

from helpers import channel_block_grid, closed_box_grid, mixed_bc_grid, periodic2d_grid, rel_err
from nabla_b200 import cases

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_small.npz"))
HAVE_REF = os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                       "libnabla_ref.so"))


def test_restatement_apply_a_matches_golden(orc):
    g = mixed_bc_grid()
    assert np.array_equal(g.solid, GOLD["applyA_mixed_solid"])
    got = orc.apply_a(g, GOLD["applyA_mixed_x"])
    assert rel_err(got, GOLD["applyA_mixed_Ax"]) < 1e-14


@pytest.mark.parametrize("name,grid,tol", [("mg_channel", channel_block_grid, 1e-10),
                                           ("mg_periodic", lambda: periodic2d_grid(24), 1e-12)])
def test_restatement_mg_matches_golden(orc, name, grid, tol):
    g = grid()
    x, rep = orc.poisson(g, GOLD[f"{name}_b"], tol, 100)
    it, res, conv = GOLD[f"{name}_rep"]
    assert rep.iterations == int(it)
    assert rep.converged == int(conv)
    assert abs(rep.residual - res) <= 1e-3 * res + 1e-15
    assert rel_err(x, GOLD[f"{name}_x"]) < 1e-10


def test_restatement_mg_box_with_solids(orc):
    g = closed_box_grid()
    assert np.array_equal(g.solid, GOLD["mg_box_solid"])
    x, rep = orc.poisson(g, GOLD["mg_box_b"], 1e-10, 100)
    assert rep.iterations == int(GOLD["mg_box_rep"][0])
    assert rel_err(x, GOLD["mg_box_x"]) < 1e-10


def test_reference_test_expectations_on_restatement(orc):
    """core/tests/test_flow.cpp:63-117: converged, residual < 1e-8, <= 50 cycles,
    RMS error vs the manufactured solution < 1e-6."""
    g = channel_block_grid()
    x, rep = orc.poisson(g, GOLD["mg_channel_b"], 1e-10, 100)
    assert rep.converged and rep.residual < 1e-8 and rep.iterations <= 50
    assert np.sqrt(np.mean((x - GOLD["mg_channel_xexact"]) ** 2)) < 1e-6


def test_restatement_tgv_steps_match_golden(orc):
    g, cfg = cases.taylor_green(16)
    ns = orc.ns(g, cfg)
    ns.set_state(*cases.taylor_green_state(g))
    dt = ns.compute_dt()
    assert dt == pytest.approx(float(GOLD["tgv16_dt"]), rel=1e-15)
    for s in (1, 2):
        r = ns.step(dt)
        for f, a in zip("uvwp", ns.get_state()):
            assert rel_err(a, GOLD[f"tgv16_s{s}_{f}"]) < 1e-12, (s, f)
        assert r.poisson_iters == int(GOLD[f"tgv16_s{s}_rep"][0])


def test_restatement_cube_steps_match_golden(orc):
    g, cfg = cases.wall_mounted_cube(2, 200.0)
    ns = orc.ns(g, cfg)
    ns.initialize()
    for s in (1, 2):
        r = ns.step()
        for f, a in zip("uvwp", ns.get_state()):
            assert rel_err(a, GOLD[f"cube2_s{s}_{f}"]) < 1e-12, (s, f)
        dt, iters, cd, cl, mass = GOLD[f"cube2_s{s}_rep"]
        assert r.dt == pytest.approx(dt, rel=1e-14)
        assert r.poisson_iters == int(iters)
        assert r.cd == pytest.approx(cd, rel=1e-9, abs=1e-12)


def test_morton_known_answers(orc):
    """core/tests/test_morton.cpp:26-39 bit patterns and golden random keys."""
    assert orc.morton_encode(1, 0, 0) == 1
    assert orc.morton_encode(0, 1, 0) == 2
    assert orc.morton_encode(0, 0, 1) == 4
    for (x, y, z), k in zip(GOLD["morton_coords"], GOLD["morton_keys"]):
        assert orc.morton_encode(int(x), int(y), int(z)) == int(k)


@pytest.mark.skipif(not HAVE_REF, reason="reference library not built")
@pytest.mark.parametrize("builder", ["lid", "channel"])
def test_restatement_matches_live_reference_2d(orc, ref, builder):
    if builder == "lid":
        g, cfg = cases.lid_cavity(12, 100.0)
    else:
        g, cfg = cases.channel(24, 8, 100.0)
        cfg.convection = 1
    a, b = orc.ns(g, cfg), ref.ns(g, cfg)
    a.initialize()
    b.initialize()
    for _ in range(3):
        ra, rb = a.step(), b.step()
        assert ra.poisson_iters == rb.poisson_iters
    for x, y in zip(a.get_state(), b.get_state()):
        assert rel_err(x, y) < 1e-12


@pytest.mark.skipif(not HAVE_REF, reason="reference library not built")
def test_restatement_matches_live_reference_mixed_bc(orc, ref):
    g = mixed_bc_grid()
    cfg = cases.flow_config(reynolds=50.0, convection=1, poisson_tol=1e-10)
    a, b = orc.ns(g, cfg), ref.ns(g, cfg)
    a.initialize()
    b.initialize()
    for _ in range(2):
        ra, rb = a.step(), b.step()
        assert ra.poisson_iters == rb.poisson_iters
    for x, y in zip(a.get_state(), b.get_state()):
        assert rel_err(x, y) < 1e-11
