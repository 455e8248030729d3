"""GPU solver against the oracle (FP64 path).

The oracle runs in its correctly-rounded mode (x^(-1/2) evaluated as the GPU evaluates it; in its
default mode it is pinned bit for bit to the reference solver, tests/test_oracle_golden.py).  With
that single substitution the GPU's FP64 step keeps the reference's operation order everywhere, so
every compared quantity must be bit-identical: node kinematics, forces, rigid-body state, works and
the contact list (candidates, active set, inherited history)."""
import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice

pytestmark = pytest.mark.gpu

CONTACT_INT = ["bodyS", "borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM", "nb_internal"]
CONTACT_DBL = ["gapn", "vgapn", "gapt", "vgapt", "xsi", "xnorm", "ynorm", "xtan", "ytan", "effective_mass", "length",
               "fx", "fy"]


def assert_contacts_equal(a, b):
    assert len(a) == len(b), f"contact counts differ: {len(a)} vs {len(b)}"
    for k in CONTACT_INT:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in ("nodeM", "shiftMk"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in CONTACT_DBL + ["shapeM", "internal"]:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def make_pair(nx=3, ny=3):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_of(squeezed_lattice(nx, ny))
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    return g, o


def test_setup_proximity_identical(gpu_lib, oracle_built):
    g, o = make_pair()
    assert_contacts_equal(g.contacts(), o.contacts())
    np.testing.assert_array_equal(g.positions(), o.positions())


def test_one_step_forces_identical(gpu_lib, oracle_built):
    g, o = make_pair()
    g.record_forces(True)
    g.step(1)
    o.step(1)
    fg, fo = g.forces(), o.forces()
    for k in ("internal", "contact", "neumann", "dirichlet", "total"):
        np.testing.assert_array_equal(fg[k], fo[k], err_msg=k)
    np.testing.assert_array_equal(g.node_state(), o.node_state())
    rg, rfg = g.rigid()
    ro, rfo = o.rigid()
    np.testing.assert_array_equal(rg, ro)
    np.testing.assert_array_equal(rfg, rfo)


@pytest.mark.parametrize("nsteps", [40, 200])
def test_trajectory_identical(gpu_lib, oracle_built, nsteps):
    g, o = make_pair()
    for _ in range(nsteps // 20):
        g.step(20)
        o.step(20)
        np.testing.assert_array_equal(g.node_state(), o.node_state())
        assert_contacts_equal(g.contacts(), o.contacts())
    np.testing.assert_array_equal(g.positions(), o.positions())
    np.testing.assert_array_equal(g.rigid()[0], o.rigid()[0])
    np.testing.assert_array_equal(g.works(), o.works())
    assert g.error_words()[2] == 0 and o.stale_shape_events() == 0
    assert (g.contacts()["fx"] != 0).sum() > 0, "scenario must have active contacts"


def test_proximity_from_uploaded_state(gpu_lib, oracle_built):
    """Candidate lists are rebuilt bit-identically from identical positions: the oracle's state after
    120 steps (kinematics, rigid bodies, contact list with history) is uploaded to the GPU, both take
    one step and then run Update_proximity on the resulting positions."""
    g, o = make_pair()
    o.step(120)
    g.set_node_state(o.node_state())
    g.set_rigid(o.rigid()[0])
    g.set_contacts(o.contacts())
    g.set_time(o.time, o.dt, o.time + 100 * o.dt)
    g.step(1, proximity=False)
    o.step(1, proximity=False)
    np.testing.assert_array_equal(g.node_state(), o.node_state())
    g.update_proximity()
    o.update_proximity()
    assert_contacts_equal(g.contacts(), o.contacts())


@pytest.mark.parametrize("seed", [5, 11])
def test_biaxial_sample_identical(gpu_lib, oracle_built, seed):
    """Small biaxial sample: long rigid plate and wall borders (segment-block pruning of the master
    search), self contact, rigid-rigid pairs under the inert law, incoming ranges from many senders,
    60 proximity updates."""
    from melody2d_b200 import generator as gen
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = gen.flatten(gen.biaxial_scene(seed=seed, n_discs=12, n_border=32, n_interior=80, workers=1))
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    assert_contacts_equal(g.contacts(), o.contacts())
    for _ in range(12):
        g.step(50)
        o.step(50)
        np.testing.assert_array_equal(g.node_state(), o.node_state())
        assert_contacts_equal(g.contacts(), o.contacts())
    np.testing.assert_array_equal(g.rigid()[0], o.rigid()[0])
    np.testing.assert_array_equal(g.works(), o.works())
    assert (g.contacts()["fx"] != 0).sum() > 0
    g.close()
