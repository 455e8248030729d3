"""The cell-list broad phase of Update_proximity (hashed uniform grid, counting sort by bucket; big
boxes such as walls and plates kept out of the grid) must give the neighbour lists of the all-pairs
pass (Code/Proximity.h:112-169) entry for entry.  Models of at least MELGPU_CELL_MIN_BODIES bodies
use it (64 by default, so the 2000-disc workload of tests/test_gpu_configs.py runs it); here the
threshold is lowered to 0 so that small cases run it too: an x-periodic domain with seams crossed
by contacts, a biaxial sample with long walls, and a pressed lattice.  After every stretch of steps
with proximity updates the contact list, node state and contact pressures equal the
correctly-rounded oracle's bit for bit, and the same model on the all-pairs pass."""
import numpy as np
import pytest

from test_gpu_parity import assert_contacts_equal

pytestmark = pytest.mark.gpu


def scene_of(case):
    from melody2d_b200 import generator as g
    if case == "periodic":
        return g.periodic_strip_scene()
    if case == "biaxial12":
        return g.biaxial_scene(seed=5, n_discs=12, n_border=32, n_interior=80, workers=1)
    return g.disc_lattice_scene(seed=0, nx=3, ny=3, pitch=2.0e-3, gap0=-1e-6, nsteps=300, v_plate=0.05)


@pytest.mark.parametrize("case", ["periodic", "biaxial12", "lattice"])
def test_cell_list_equals_all_pairs_and_oracle(gpu_lib, oracle_built, case, monkeypatch):
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = g.flatten(scene_of(case))
    monkeypatch.setenv("MELGPU_CELL_MIN_BODIES", "0")
    cell = Solver.from_flat(flat)
    monkeypatch.setenv("MELGPU_CELL_MIN_BODIES", "1000000000")
    pairs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    assert_contacts_equal(cell.contacts(), o.contacts())
    for _ in range(6):
        for s in (cell, pairs, o):
            s.step(50)
        assert_contacts_equal(cell.contacts(), o.contacts())
        assert_contacts_equal(cell.contacts(), pairs.contacts())
        np.testing.assert_array_equal(cell.node_state(), o.node_state())
        np.testing.assert_array_equal(cell.contact_pressures(), o.contact_pressures())
    c = cell.contacts()
    assert len(c["fx"]) > 0 and ((c["fx"] != 0) | (c["fy"] != 0)).sum() > 0
    if case == "periodic":
        assert set(np.unique(c["shiftM"]).tolist()) >= {-1, 0, 1}
    cell.close()
    pairs.close()
