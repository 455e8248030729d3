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


def _reduce_static(L, vel, mass, disp, n, cont, nc, out, stream):
    return L.mel_monitor_reduce_static(ctypes.c_void_p(vel.data_ptr()), ctypes.c_void_p(mass.data_ptr()),
                                       ctypes.c_void_p(disp.data_ptr()), n, ctypes.c_void_p(cont.data_ptr()), nc,
                                       ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


@pytest.mark.parametrize("n_nodes,n_contacts", [(300_001, 123_457), (2_097_152, 2_097_152)])
def test_static_scratch_many_blocks(gpu_lib, n_nodes, n_contacts):
    """Sizes that spread the reduction over many blocks, up to the largest accepted size (1024 blocks
    of partials), against a float64 reduction in numpy.  The values are positive so that the sums
    carry no cancellation and the order of the additions only moves the last bits."""
    import torch
    from melody2d_b200.abi import CONTACT_DTYPE
    from melody2d_b200.solver import lib
    rng = np.random.default_rng(n_nodes)
    v = rng.uniform(0.5, 1.5, (n_nodes, 2))
    m = rng.uniform(1e-6, 2e-6, (n_nodes, 2))
    u = rng.uniform(1e-5, 3e-5, (n_nodes, 2))
    cont = np.zeros(n_contacts, dtype=CONTACT_DTYPE)
    act = rng.random(n_contacts) < 0.3
    cont["fx"][act] = rng.uniform(-1., 1., int(act.sum()))
    only_y = (~act) & (rng.random(n_contacts) < 0.1)      # a force along y alone also counts as active
    cont["fy"][only_y] = 1e-3
    ke = float(np.sum(0.5 * v[:, 0] * v[:, 0] * m[:, 0] + 0.5 * v[:, 1] * v[:, 1] * m[:, 1]))
    ux = float(np.sum(u[:, 0] * m[:, 0]) / np.sum(m[:, 0]))
    uy = float(np.sum(u[:, 1] * m[:, 1]) / np.sum(m[:, 0]))
    n_act = int(act.sum() + only_y.sum())
    dev = torch.device("cuda", 0)
    tv, tm, tu = (torch.from_numpy(a).to(dev) for a in (v, m, u))
    tc = torch.from_numpy(cont.view(np.uint8).reshape(-1)).to(dev)
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = lib()
    res = []
    for _ in range(2):
        out.fill_(-1.)
        assert _reduce_static(L, tv, tm, tu, n_nodes, tc, n_contacts, out, stream) == 0, L.mel_last_error_string()
        torch.cuda.synchronize(dev)
        res.append(out.cpu().numpy().copy())
    for r in res:
        np.testing.assert_allclose(r[0], ke, rtol=1e-12)
        np.testing.assert_allclose(r[1], ux, rtol=1e-12)
        np.testing.assert_allclose(r[2], uy, rtol=1e-12)
        assert int(r[3]) == n_act
    np.testing.assert_array_equal(res[0], res[1])


def test_static_scratch_rejects_oversize(gpu_lib):
    from melody2d_b200.solver import lib
    L = lib()
    rc = L.mel_monitor_reduce_static(None, None, None, 2_097_153, None, 0, ctypes.c_void_p(1), None)
    assert rc == 1
    assert b"at most" in L.mel_last_error_string()
