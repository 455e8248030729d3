"""Chunk images (the body kernel's Gauss-point input) checked on the CPU: a model of the kernel's
Gauss-point pass (tests/emul/chunk_emul.cpp, same image parsing and index arithmetic as the CUDA
code, every followed index bounds-checked) must reproduce the oracle's internal forces bit for
bit, at every chunk size the build may choose."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, flat_of, squeezed_lattice


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("emul") / "libchunkemul.so")
    csrc = os.path.join(ROOT, "melody2d_b200", "csrc")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I" + csrc,
           "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "emul", "chunk_emul.cpp"), os.path.join(csrc, "mel_chunks.cpp"), "-o", out]
    subprocess.run(cmd, check=True)
    L = C.CDLL(out)
    L.emul_internal_forces.restype = C.c_int
    L.emul_internal_forces.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.emul_error.restype = C.c_char_p
    return L


@pytest.mark.parametrize("ecap", [2048, 1024, 256])
def test_chunk_pass_matches_oracle(emul, oracle_built, ecap):
    from melody2d_b200.abi import Desc
    from oracle.pyoracle import Oracle
    flat = flat_of(squeezed_lattice(3, 3))
    o = Oracle(flat)
    o.step(30)
    up = np.ascontiguousarray(o.node_state()[:, 6:8]).copy()   # displacements the next pass reads
    o.step(1)
    ref = o.forces()["internal"]
    desc = Desc(flat)
    f = np.zeros_like(up)
    stats = np.zeros(4, dtype=np.int64)
    rc = emul.emul_internal_forces(C.byref(desc.desc), ecap, up.ctypes.data, f.ctypes.data, stats.ctypes.data)
    assert rc == 0, (rc, emul.emul_error())
    assert stats[0] > 0 and stats[3] % 16 == 0
    # padding: point groups padded to their widest slot, and each chunk rounded to 8 entries
    assert stats[2] < 0.2 * stats[1], "padding above a fifth of the stored entries"
    np.testing.assert_array_equal(f, ref)
    assert np.abs(ref).max() > 0


@pytest.mark.parametrize("ecap", [3584, 2048, 1024, 256])
def test_segmented_pull_layout(emul, ecap):
    """Images of the mixed pass's two-buffer loop: the pull pieces list every stored entry once,
    each piece's entries are stored for its node, a node's pieces belong to one of the seven pull
    warps, and the piece sums give the nodal forces of a direct scatter."""
    from melody2d_b200.abi import Desc
    flat = flat_of(squeezed_lattice(3, 3))
    desc = Desc(flat)
    rng = np.random.default_rng(5)
    up = rng.standard_normal((len(flat["node_x0"]) // 2, 2)) * 1e-5
    f_list = np.zeros_like(up)
    f_direct = np.zeros_like(up)
    stats = np.zeros(4, dtype=np.int64)
    emul.emul_segmented_pull.restype = C.c_int
    emul.emul_segmented_pull.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = emul.emul_segmented_pull(C.byref(desc.desc), ecap, up.ctypes.data, f_list.ctypes.data,
                                  f_direct.ctypes.data, stats.ctypes.data)
    assert rc == 0, (rc, emul.emul_error())
    assert stats[0] > 0 and stats[1] > 0
    # the heaviest warp's share of the entries stays near the mean (whole nodes only)
    assert stats[3] < 1500, stats
    scale = np.abs(f_direct).max()
    assert scale > 0
    np.testing.assert_allclose(f_list, f_direct, rtol=0, atol=1e-12 * scale)


def wide_scene():
    """Two discs of 4,360 nodes each (above the 4,096 a body's shared memory holds) between plates
    and walls: their images carry the 16-bit node section."""
    from melody2d_b200 import generator as g
    return g.biaxial_scene(seed=3, n_discs=2, n_border=160, n_interior=4200, workers=1)


def test_chunk_pass_wide_bodies_match_oracle(emul, oracle_built):
    """The FP64 images of bodies above 4,096 nodes name each pull slot's node in a 16-bit section;
    the CPU model of the kernel's chunk pass reproduces the oracle's internal forces bit for bit."""
    from melody2d_b200 import generator as g
    from melody2d_b200.abi import Desc
    from oracle.pyoracle import Oracle
    flat = g.flatten(wide_scene())
    assert np.diff(flat["body_node_ptr"]).max() > 4096
    o = Oracle(flat)
    # a seeded field of displacement parameters (the sample is barely loaded after a few steps)
    st = o.node_state()
    deform = np.repeat(np.asarray(flat["body_type"]) == 0, np.diff(flat["body_node_ptr"]))
    st[deform, 6:8] = np.random.default_rng(8).standard_normal((int(deform.sum()), 2)) * 1e-7
    o.set_node_state(st)
    up = np.ascontiguousarray(st[:, 6:8]).copy()
    o.step(1, proximity=False)
    ref = o.forces()["internal"]
    desc = Desc(flat)
    f = np.zeros_like(up)
    stats = np.zeros(4, dtype=np.int64)
    rc = emul.emul_internal_forces(C.byref(desc.desc), 2048, up.ctypes.data, f.ctypes.data, stats.ctypes.data)
    assert rc == 0, (rc, emul.emul_error())
    np.testing.assert_array_equal(f, ref)
    assert np.abs(ref).max() > 0


def test_segmented_pull_wide_bodies(emul):
    """Mixed images of bodies above 4,096 nodes: pieces carry 16-bit nodes."""
    from melody2d_b200 import generator as g
    from melody2d_b200.abi import Desc
    flat = g.flatten(wide_scene())
    desc = Desc(flat)
    rng = np.random.default_rng(6)
    up = rng.standard_normal((len(flat["node_x0"]) // 2, 2)) * 1e-5
    f_list = np.zeros_like(up)
    f_direct = np.zeros_like(up)
    stats = np.zeros(4, dtype=np.int64)
    emul.emul_segmented_pull.restype = C.c_int
    emul.emul_segmented_pull.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = emul.emul_segmented_pull(C.byref(desc.desc), 3328, up.ctypes.data, f_list.ctypes.data,
                                  f_direct.ctypes.data, stats.ctypes.data)
    assert rc == 0, (rc, emul.emul_error())
    scale = np.abs(f_direct).max()
    np.testing.assert_allclose(f_list, f_direct, rtol=0, atol=1e-12 * scale)
