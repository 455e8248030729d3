"""Mixed-precision form (dN, strain, stress and contributions in FP32; positions, velocities,
contact geometry and nodal force sums in FP64) against the FP64 oracle.

Stated tolerances, relative to the oracle: kinetic energy, wall reaction (contact force and
driven-DOF reaction of the rigid plates) and mass-weighted mean displacement within 1e-5 after
1000 steps; the active-contact count equal; internal nodal forces of one step from the oracle's
state within 1e-5 of the largest force."""
import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def monitored(m):
    return (m.kinetic_energy, np.array(list(m.mean_displacement)), np.array(list(m.rigid_force)),
            np.array(list(m.rigid_dirichlet)), m.active_contacts)


def scenes():
    from melody2d_b200 import generator as g
    yield "lattice3x3", flat_of(squeezed_lattice(3, 3))
    yield "biaxial12", g.flatten(g.biaxial_scene(seed=5, n_discs=12, n_border=32, n_interior=80, workers=1))


@pytest.mark.parametrize("case", ["lattice3x3", "biaxial12"])
def test_mixed_monitored_quantities(gpu_lib, oracle_built, case):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = dict(scenes())[case]
    g = Solver.from_flat(flat, precision=1)
    o = Oracle(flat, correctly_rounded=True)
    for _ in range(5):
        g.step(200)
        o.step(200)
        ke_g, u_g, rf_g, rd_g, act_g = monitored(g.monitor())
        ke_o, u_o, rf_o, rd_o, act_o = monitored(o.monitor())
        assert rel(ke_g, ke_o) <= TOL, ("kinetic energy", rel(ke_g, ke_o))
        assert rel(u_g, u_o) <= TOL, ("mean displacement", rel(u_g, u_o))
        assert rel(rf_g, rf_o) <= TOL, ("wall contact force", rel(rf_g, rf_o))
        assert rel(rd_g, rd_o) <= TOL, ("wall reaction", rel(rd_g, rd_o))
        assert act_g == act_o
    assert act_o > 0
    g.close()


def test_mixed_internal_forces_one_step(gpu_lib, oracle_built):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_of(squeezed_lattice(3, 3))
    o = Oracle(flat, correctly_rounded=True)
    o.step(30)
    g = Solver.from_flat(flat, precision=1)
    g.set_node_state(o.node_state())
    g.set_rigid(o.rigid()[0])
    g.set_contacts(o.contacts())
    g.set_time(o.time, o.dt, o.time + 100 * o.dt)
    g.record_forces(True)
    g.step(1, proximity=False)
    o.step(1, proximity=False)
    fg, fo = g.forces()["internal"], o.forces()["internal"]
    assert np.abs(fg - fo).max() <= TOL * np.abs(fo).max()
    assert not np.array_equal(fg, fo), "the mixed form must actually run in FP32"
    g.close()
