"""Failure detection on the GPU without a GPU fault: the body kernel's pipeline waits are bounded
(1 s), and a wait that gives up makes the kernel set an error word, let its copies in flight land
(a separate bounded wait) and return, so that the step reports MEL_ERR_TIMEOUT and the context
stays usable.  The environment variable MELGPU_WAIT_NS, read when a model is created, shortens the
bound; at 0 a wait only tests the barrier once, so the first chunk a body waits for is not there
yet and the wait gives up."""
import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice

pytestmark = pytest.mark.gpu


def test_pipeline_wait_gives_up_and_context_survives(gpu_lib, oracle_built, monkeypatch):
    from melody2d_b200.solver import MelError, Solver
    from oracle.pyoracle import Oracle
    flat = flat_of(squeezed_lattice(3, 3))
    monkeypatch.setenv("MELGPU_WAIT_NS", "0")
    s = Solver.from_flat(flat)
    with pytest.raises(MelError) as e:
        s.step(1)
    assert e.value.code == 7, str(e.value)                  # MEL_ERR_TIMEOUT
    assert s.error_words()[6] != 0                          # MEL_E_WAIT
    s.close()
    monkeypatch.delenv("MELGPU_WAIT_NS")
    # same process, same device: a fresh model steps normally and matches the oracle
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    g.step(20)
    o.step(20)
    np.testing.assert_array_equal(g.node_state(), o.node_state())
    g.close()
