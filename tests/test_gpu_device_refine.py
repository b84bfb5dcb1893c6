"""Refinement on the device (nb_amr_refine_device, nb_amr_case_refine): the
split of flagged leaves with 26-neighbour 2:1 balance restored by rounds of
device binary searches in the sorted keys, and the ranking of the new leaves
by a device sort, must give exactly the host maps' leaf list (nb_amr_refine,
itself checked against the reference's Octree through the map parity tests),
integer for integer in rank order: on random refinement storms with walls and
with periodic wrap, on the obstacle channel, and from a case's own device
sensors. A regrid pass on the device equals the host regrid pass."""
import numpy as np
import pytest

from nabla_b200 import abi, amr, workloads

pytestmark = pytest.mark.gpu


def _ranked(geom, leaves):
    return amr.tree_maps(geom, leaves)[1]


@pytest.mark.parametrize("periodic", [False, True])
def test_device_refinement_equals_host(ctx, periodic):
    bc = abi.BC_PERIODIC if periodic else abi.BC_WALL
    g = amr.make_geom((3, 2, 2), (0.1, 0.1, 0.1), 3, [dict(type=bc) for _ in range(6)])
    rng = np.random.default_rng(12345 + periodic)
    lv = amr.base_leaves([3, 2, 2])
    for _ in range(4):
        flags = (rng.random(len(lv)) < 0.2).astype(np.uint8)
        host = amr.refine(g, lv, flags)
        dev = amr.refine_device(g, lv, flags, ctx)
        assert np.array_equal(dev, _ranked(g, host))
        lv = host
    assert lv[:, 0].max() == 3


def test_device_refinement_of_channel_mesh(ctx):
    w = workloads.obstacle_channel(0)
    flags = (np.random.default_rng(5).random(len(w.leaves)) < 0.1).astype(np.uint8)
    host = amr.refine(w.geom, w.leaves, flags)
    dev = amr.refine_device(w.geom, w.leaves[::-1].copy(), flags[::-1].copy(), ctx)
    assert np.array_equal(dev, _ranked(w.geom, host))


def _refinable_case():
    """A 2-level Taylor-Green box with solids whose geometry allows one more level."""
    t = workloads.tgv_box_case(0)
    t.geom.lmax += 1
    return t


def test_case_refinement_from_device_sensors(ctx):
    t = _refinable_case()
    mesh = amr.AmrMesh(t.geom, t.leaves, solid=t.solid, ctx=ctx)
    case = amr.AmrCase(mesh, t.config)
    case.set_state(*t.initial_state(case))
    s = case.sensors()[:, 0]
    above = float(np.percentile(s, 70))
    host = amr.refine(t.geom, mesh.leaves, ((s > above) & (mesh.leaves[:, 0] < t.geom.lmax)).astype(np.uint8))
    dev = case.refine_leaves(0, above)
    assert len(dev) > len(mesh.leaves)
    assert np.array_equal(dev, _ranked(t.geom, host))
    case.close()
    mesh.close()


def test_device_regrid_equals_host_regrid(ctx):
    t = _refinable_case()
    mesh = amr.AmrMesh(t.geom, t.leaves, solid=t.solid, ctx=ctx)
    case = amr.AmrCase(mesh, t.config)
    case.set_state(*t.initial_state(case))
    case.step()
    s = case.sensors()[:, 0]
    thr, low = float(np.percentile(s, 60)), float(np.percentile(s, 10))
    a = amr.regrid(case, thr, low, device=True)
    b = amr.regrid(case, thr, low, device=False)
    assert np.array_equal(a.mesh.leaves, b.mesh.leaves)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    for c in (a, b):
        c.close()
    case.close()
    mesh.close()
