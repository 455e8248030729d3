"""Asynchronous checkpoints (mel_checkpoint_start / mel_checkpoint_read).  A snapshot started
after 30 steps and read after 25 more (the copy overlaps those steps and their proximity
updates) must equal the blocking downloads taken at the moment it started, and a solver restarted
from it must continue exactly as the original did.  The same holds for a member of a batch."""
import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice
from test_gpu_parity import assert_contacts_equal

pytestmark = pytest.mark.gpu


def blocking_state(s):
    return {"node_state": s.node_state(), "rigid": s.rigid()[0], "works": s.works(), "contacts": s.contacts(),
            "time": s.time()}


def assert_snapshot(cp, ref):
    np.testing.assert_array_equal(cp["node_state"], ref["node_state"])
    np.testing.assert_array_equal(cp["rigid"].reshape(-1), ref["rigid"].reshape(-1))
    np.testing.assert_array_equal(cp["works"], ref["works"])
    assert_contacts_equal(cp["contacts"], ref["contacts"])
    assert (cp["time"], cp["dt"]) == ref["time"]


def test_checkpoint_matches_blocking_downloads_and_restarts(gpu_lib):
    from melody2d_b200.solver import Solver
    flat = flat_of(squeezed_lattice(3, 3))
    s = Solver.from_flat(flat)
    s.step(30)
    ref = blocking_state(s)
    s.checkpoint_start()
    s.step(25)
    cp = s.checkpoint_read()
    assert_snapshot(cp, ref)
    assert len(cp["contacts"]) > 0
    with pytest.raises(Exception):
        s.checkpoint_read()                 # read once per start
    r = Solver.from_flat(flat)
    r.set_node_state(cp["node_state"])
    r.set_rigid(cp["rigid"])
    r.set_contacts(cp["contacts"])
    r.set_time(cp["time"], cp["dt"], cp["next_contact_update"])
    r.step(25)
    np.testing.assert_array_equal(r.node_state(), s.node_state())
    assert_contacts_equal(r.contacts(), s.contacts())
    s.close()
    r.close()


def test_checkpoint_of_batch_member(gpu_lib):
    from melody2d_b200.solver import Batch, Solver
    a = Solver.from_flat(flat_of(squeezed_lattice(2, 2)))
    m = Solver.from_flat(flat_of(squeezed_lattice(3, 3)))
    b = Batch()
    b.admit(a)
    b.admit(m)
    b.step(30)
    ref = blocking_state(m)
    m.checkpoint_start()
    b.step(25)
    assert_snapshot(m.checkpoint_read(), ref)
    b.close()
    a.close()
    m.close()
