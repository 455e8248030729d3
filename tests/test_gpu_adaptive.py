"""Solver_step on the GPU (Code/Solver.h:98-486): Adaptive_Euler, Euler_2, Mass_Scaling and
Adaptive_Mass_Scaling on the pressed 3x3 lattice, against the oracle in its correctly-rounded mode,
bit for bit: node state (including the temporary displacements, errors and mass-scaling factors
through the state they produce), rigid bodies, works, contact list, contact pressures, Time,
Deltat and the scheme's statistics (attempts, largest and mean error, scaled masses) after 50 and
100 accepted steps.  The oracle is pinned to the compiled reference on the same four cases
(tests/test_oracle_laws.py)."""
import numpy as np
import pytest

from test_gpu_parity import assert_contacts_equal
from test_oracle_laws import SOLVER_CASES, case_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(SOLVER_CASES))
def test_solver_step_identical(gpu_lib, oracle_built, case):
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = g.flatten(case_scene(case))
    s = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    attempts = 0
    for k in range(2):
        s.step(50)
        o.step(50)
        assert s.time() == (o.time, o.dt), case
        np.testing.assert_array_equal(s.solver_stats(), o.solver_stats(), err_msg=case)
        attempts = max(attempts, int(s.solver_stats()[0]))
        np.testing.assert_array_equal(s.node_state(), o.node_state(), err_msg=case)
        np.testing.assert_array_equal(s.rigid()[0], o.rigid()[0], err_msg=case)
        np.testing.assert_array_equal(s.works(), o.works(), err_msg=case)
        assert_contacts_equal(s.contacts(), o.contacts())
        np.testing.assert_array_equal(s.contact_pressures(), o.contact_pressures(), err_msg=case)
    assert (s.contacts()["fx"] != 0).sum() > 0
    s.close()
