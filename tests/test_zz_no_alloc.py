"""mel_monitor_reduce_static: the monitored-quantity reduction for callers that cannot allocate
device memory (a framework that owns all device memory through its own allocator, or a deployment
with a fixed device-memory budget).  They hand over device arrays they already hold; the entry point
keeps its block partials in a file-scope device array instead of allocating.

Checked through the C ABI against mel_monitor_compute on the same state, on two calls in a row.
The device buffers standing for the caller's memory are made with torch in this test only.  This
file is collected last so that a stop-at-first-failure run has executed every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import flat_of, squeezed_lattice

pytestmark = pytest.mark.gpu


def test_static_scratch_reduction_matches_monitor(gpu_lib):
    import torch
    from melody2d_b200.solver import Solver, lib
    flat = flat_of(squeezed_lattice(3, 3))
    s = Solver.from_flat(flat)
    s.step(30)
    ref = s.monitor()                                    # existing entry point
    st = s.node_state()
    cont = s.contacts()
    dev = torch.device("cuda", 0)
    vel = torch.from_numpy(np.ascontiguousarray(st[:, 2:4])).to(dev)
    disp = torch.from_numpy(np.ascontiguousarray(st[:, 0:2])).to(dev)
    mass = torch.from_numpy(np.ascontiguousarray(np.asarray(flat["node_mass"]).reshape(-1, 2))).to(dev)
    cbytes = torch.from_numpy(np.frombuffer(cont.tobytes(), dtype=np.uint8).copy()).to(dev)
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = lib()
    results = []
    for _ in range(2):                                   # two calls in a row share the static array
        out.zero_()
        rc = L.mel_monitor_reduce_static(ctypes.c_void_p(vel.data_ptr()), ctypes.c_void_p(mass.data_ptr()),
                                         ctypes.c_void_p(disp.data_ptr()), s.nn, ctypes.c_void_p(cbytes.data_ptr()),
                                         len(cont), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, L.mel_last_error_string()
        torch.cuda.synchronize(dev)
        results.append(out.cpu().numpy().copy())
    for r in results:
        np.testing.assert_allclose(r[0], ref.kinetic_energy, rtol=1e-12, atol=0)
        np.testing.assert_allclose(r[1:3], list(ref.mean_displacement), rtol=1e-12, atol=1e-30)
        assert int(r[3]) == ref.active_contacts
    np.testing.assert_array_equal(results[0], results[1])
    assert ref.active_contacts > 0 and ref.kinetic_energy > 0
    s.close()


def test_static_scratch_rejects_oversize(gpu_lib):
    from melody2d_b200.solver import lib
    L = lib()
    rc = L.mel_monitor_reduce_static(None, None, None, 2_097_153, None, 0, ctypes.c_void_p(1), None)
    assert rc == 1
    assert b"at most" in L.mel_last_error_string()
