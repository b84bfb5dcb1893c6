"""Device-side regridding of octree cases: per-leaf sensors
(nb_amr_case_sensors, the velocity-gradient sensors of
core/src/adaptive/adaptive_core.cpp:96-113), the conservative state transfer
between a mesh and its refinement or coarsening (nb_amr_case_transfer), and a
full regrid pass (amr.regrid) after which the case keeps stepping."""
import numpy as np
import pytest

from amr_helpers import closed_box_geom, refine_where, two_level_leaves
from nabla_b200 import abi, amr, cases

pytestmark = pytest.mark.gpu


def _cfg():
    return cases.flow_config(reynolds=100.0, convection=abi.CONV_WENO5, poisson_tol=1e-10)


def test_sensors_of_a_shear_flow(ctx):
    geom = closed_box_geom()
    mesh = amr.AmrMesh(geom, two_level_leaves(geom), ctx=ctx)
    ac = amr.AmrCase(mesh, _cfg())
    a, b = 3.0, 0.7
    y0 = ac.face_positions(0)[1]
    xc = mesh.cell_centers()[0]
    ac.set_state(a * y0, np.zeros(ac.sizes[1]), np.zeros(ac.sizes[2]), b * xc)
    s = ac.sensors()
    assert s.shape == (mesh.leaves.shape[0], 4)
    assert np.allclose(s[:, 0], a, rtol=1e-12)         # |vorticity|
    assert np.allclose(s[:, 1], a, rtol=1e-12)         # sqrt(2 S:S)
    assert np.abs(s[:, 2]).max() <= 1e-12 * a * a      # Q
    assert np.allclose(s[:, 3], b, rtol=1e-12)         # |grad p|


def _linear_state(ac):
    """Each velocity component varies along its own axis only, divergence free."""
    x = ac.face_positions(0)[0]
    y = ac.face_positions(1)[1]
    z = ac.face_positions(2)[2]
    return 1.0 + 0.5 * x, 2.0 - 0.25 * y, 0.3 - 0.25 * z


def test_transfer_to_the_same_mesh_is_a_copy(ctx):
    geom = closed_box_geom()
    mesh = amr.AmrMesh(geom, two_level_leaves(geom), ctx=ctx)
    a, b = amr.AmrCase(mesh, _cfg()), amr.AmrCase(mesh, _cfg())
    rng = np.random.default_rng(3)
    a.set_state(*[rng.uniform(-1, 1, n) for n in a.sizes])
    b.transfer_from(a)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


def test_transfer_across_refinement_and_back(ctx):
    geom = closed_box_geom()
    coarse_leaves = two_level_leaves(geom)
    fine_leaves = refine_where(geom, coarse_leaves, lambda L, x, y, z: L == 0 and x == 1 and y == 1)
    coarse = amr.AmrCase(amr.AmrMesh(geom, coarse_leaves, ctx=ctx), _cfg())
    fine = amr.AmrCase(amr.AmrMesh(geom, fine_leaves, ctx=ctx), _cfg())
    u, v, w = _linear_state(coarse)
    p = np.random.default_rng(4).uniform(-1, 1, coarse.sizes[3])
    coarse.set_state(u, v, w, p)
    fine.transfer_from(coarse)
    uf, vf, wf, pf = fine.get_state()
    for got, want in zip((uf, vf, wf), _linear_state(fine)):
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    back = amr.AmrCase(amr.AmrMesh(geom, amr.coarsen(geom, fine_leaves, np.ones(len(fine_leaves), np.uint8)),
                                   ctx=ctx), _cfg())
    # coarsening everything also merges the original level-1 octet: compare on the common mesh
    again = amr.AmrCase(coarse.mesh, _cfg())
    again.transfer_from(fine)
    for x, y in zip(again.get_state(), coarse.get_state()):
        assert np.abs(x - y).max() <= 1e-14 * max(np.abs(y).max(), 1.0)
    back.transfer_from(fine)
    for got, want in zip(back.get_state()[:3], _linear_state(back)):
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_transfer_rejects_meshes_two_levels_apart(ctx):
    geom = closed_box_geom(lmax=2)
    base = amr.base_leaves(list(geom.nb0))
    one = amr.refine(geom, base, np.ones(len(base), np.uint8))
    two = amr.refine(geom, one, np.ones(len(one), np.uint8))
    a = amr.AmrCase(amr.AmrMesh(geom, base, ctx=ctx), _cfg())
    b = amr.AmrCase(amr.AmrMesh(geom, two, ctx=ctx), _cfg())
    from nabla_b200.solver import NablaError
    with pytest.raises(NablaError, match="more than one level"):
        b.transfer_from(a)


def test_regrid_pass_keeps_stepping(ctx):
    n = 4
    h = 2 * np.pi / (8 * n)
    faces = [dict(type=abi.BC_PERIODIC) for _ in range(6)]
    geom = amr.make_geom((n, n, n), (h, h, h), 1, faces)
    mesh = amr.AmrMesh(geom, amr.base_leaves((n, n, n)), ctx=ctx)
    cfg = cases.flow_config(reynolds=1600.0, convection=abi.CONV_WENO5, poisson_tol=1e-10, cfl=0.4)
    ac = amr.AmrCase(mesh, cfg)
    st = []
    for a in range(3):
        x, y, z = ac.face_positions(a)
        st.append(np.sin(x) * np.cos(y) * np.cos(z) if a == 0 else
                  (-np.cos(x) * np.sin(y) * np.cos(z) if a == 1 else np.zeros_like(x)))
    st.append(np.zeros(ac.sizes[3]))
    ac.set_state(*st)
    ac.step(0.05)
    s = ac.sensors()[:, 0]
    fine = amr.regrid(ac, refine_above=np.quantile(s, 0.75), coarsen_below=0.0)
    assert fine.mesh.leaves.shape[0] > mesh.leaves.shape[0]
    for _ in range(2):
        rep = fine.step(0.05)
        assert rep.converged and rep.divergence_max <= 1e-8
    back = amr.regrid(fine, refine_above=np.inf, coarsen_below=np.inf)
    assert back.mesh.leaves.shape[0] == mesh.leaves.shape[0]
    rep = back.step(0.05)
    assert rep.converged and rep.divergence_max <= 1e-8
