"""Batches (mel_batch_*): several independent samples advanced by shared launches.  A sample's
state after batched steps must be bit-identical to the same sample stepped alone -- with samples
of different sizes, kinds and time steps in the mix, one admitted part-way, one retired and then
stepped alone -- since every sample runs the one-model code on its own arrays."""
import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice

pytestmark = pytest.mark.gpu


def samples():
    from melody2d_b200 import generator as g
    return [flat_of(squeezed_lattice(2, 2)), flat_of(squeezed_lattice(3, 3)),
            g.flatten(g.biaxial_scene(seed=5, n_discs=12, n_border=32, n_interior=80, workers=1))]


def state(s):
    c = s.contacts()
    return (s.node_state(), s.rigid()[0], s.works(), c.tobytes(), s.time())


def assert_same(a, b):
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)
    assert a[3] == b[3], "contact lists differ"
    assert a[4] == b[4]


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_alone(gpu_lib, precision):
    from melody2d_b200.solver import Batch, Solver
    flats = samples()
    alone = [Solver.from_flat(f, precision=precision) for f in flats]
    mixed = [Solver.from_flat(f, precision=precision) for f in flats]
    b = Batch(precision=precision)
    b.admit(mixed[0])
    b.admit(mixed[1])
    b.step(40)                      # sample 2 joins after 40 steps of the others
    b.admit(mixed[2])
    b.step(130)
    for s, n in zip(alone, (170, 170, 130)):
        s.step(n)
    for s, t in zip(alone, mixed):
        assert_same(state(s), state(t))
    # retire sample 0 and carry on with it alone; the rest keep running in the batch
    b.retire(mixed[0])
    mixed[0].step(60)
    b.step(60)
    for s in alone:
        s.step(60)
    for s, t in zip(alone, mixed):
        assert_same(state(s), state(t))
    st = b.stats()
    assert st["members"] == 2 and st["launches"] >= 3 * 60
    assert (mixed[2].contacts()["fx"] != 0).sum() > 0
    b.close()


def test_batch_member_cannot_step_alone(gpu_lib):
    from melody2d_b200.solver import Batch, MelError, Solver
    s = Solver.from_flat(flat_of(squeezed_lattice(2, 2)))
    b = Batch()
    b.admit(s)
    with pytest.raises(MelError):
        s.step(1)
    with pytest.raises(MelError):
        Batch(precision=1).admit(s)
    b.close()
    s.step(1)                       # free again once the batch is gone


def test_diverged_member_leaves_batch(gpu_lib):
    """A member whose state runs away (one border node's parameter moved 1 km: finite values, and
    no kernel derives an index from a position) is reported by its next proximity update and
    leaves the batch; the other members carry on exactly as they would alone."""
    from melody2d_b200.abi import MEL_ERR_NAN
    from melody2d_b200.solver import Batch, Solver
    flats = samples()
    alone = [Solver.from_flat(f) for f in flats]
    mixed = [Solver.from_flat(f) for f in flats]
    b = Batch()
    for s in mixed:
        b.admit(s)
    b.step(40)
    st = mixed[1].node_state()
    st[5, 6] += 1.0e3                       # nodal parameter up x of one border node
    mixed[1].set_node_state(st)
    failed = b.step(30)
    assert failed == [mixed[1]]
    code, msg = mixed[1].health()
    assert code == MEL_ERR_NAN and ("periods" in msg or "non-finite" in msg), msg
    assert b.stats()["members"] == 2
    for i in (0, 2):
        alone[i].step(70)
        assert_same(state(alone[i]), state(mixed[i]))
    b.close()
