"""Deformable bodies above 4,096 nodes: their node arrays do not fit the body kernel's shared memory,
so the kernel keeps them in global memory (displacement parameters read in place, force sums in a
scratch area) while the chunk images still stream through shared memory, and the pull names its
nodes with 16 bits.  Two discs of 4,360 nodes between plates and walls, started from a seeded field
of displacement parameters so that they vibrate from the first step: the FP64 path equals the
correctly-rounded oracle bit for bit (node state, contacts, works) over 120 steps with proximity
updates, and the mixed path stays within the mixed form's tolerance of it."""
import numpy as np
import pytest

from test_gpu_parity import assert_contacts_equal

pytestmark = pytest.mark.gpu


def wide_flat():
    from melody2d_b200 import generator as g
    flat = g.flatten(g.biaxial_scene(seed=3, n_discs=2, n_border=160, n_interior=4200, workers=1))
    assert np.diff(flat["body_node_ptr"]).max() > 4096
    return flat


def seeded_state(flat, st):
    deform = np.repeat(np.asarray(flat["body_type"]) == 0, np.diff(flat["body_node_ptr"]))
    st = st.copy()
    st[deform, 6:8] = np.random.default_rng(8).standard_normal((int(deform.sum()), 2)) * 1e-7
    return st


def test_large_bodies_fp64_bit_identical(gpu_lib, oracle_built):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = wide_flat()
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    st = seeded_state(flat, o.node_state())
    gs.set_node_state(st)
    o.set_node_state(st)
    for _ in range(3):
        gs.step(40)
        o.step(40)
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    np.testing.assert_array_equal(gs.works(), o.works())
    assert np.abs(gs.works()[:, 0]).max() > 0          # internal work: the discs deform
    gs.close()


def test_large_bodies_mixed_within_tolerance(gpu_lib):
    from melody2d_b200.solver import Solver
    flat = wide_flat()
    a = Solver.from_flat(flat, precision=0)
    m = Solver.from_flat(flat, precision=1)
    st = seeded_state(flat, a.node_state())
    a.set_node_state(st)
    m.set_node_state(st)
    a.step(120)
    m.step(120)
    sa, sm = a.node_state(), m.node_state()
    for cols in (slice(0, 2), slice(2, 4)):                 # displacements, velocities
        scale = np.abs(sa[:, cols]).max()
        assert scale > 0
        assert np.abs(sm[:, cols] - sa[:, cols]).max() <= 1e-5 * scale
    a.close()
    m.close()


def test_large_bodies_adaptive_scheme_bit_identical(gpu_lib, oracle_built):
    """Solver_step (Adaptive_Euler) with the wide bodies: both half-steps run them in their own
    launch; the state, time step and statistics equal the oracle's."""
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = wide_flat()
    flat["solver"] = 1
    sp = np.array(flat["solver_params"], dtype=np.float64)
    sp[:3] = (2e-3, 0.2, 0.9)
    flat["solver_params"] = sp
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    st = seeded_state(flat, o.node_state())
    gs.set_node_state(st)
    o.set_node_state(st)
    gs.step(40)
    o.step(40)
    np.testing.assert_array_equal(gs.node_state(), o.node_state())
    assert gs.time() == (o.time, o.dt)
    gs.close()
