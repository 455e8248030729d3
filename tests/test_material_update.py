"""UPDATE_STIFFNESS_MATRIX and UPDATE_DAMPING_MATRIX (Body::Update_material, Code/Body.h:2784-2875)
on the CPU: the library's host re-assembly (melody2d_b200/csrc/mel_material.cpp, compiled here
without CUDA) gives the MATRICES stiffness and damping entries of the oracle bit for bit, for both
material laws and each combination of the two flags.  The oracle's re-assembly is itself pinned to
the compiled reference by the update_matrices case of tests/test_oracle_laws.py."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def matlib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("mat") / "libmatemul.so")
    csrc = os.path.join(ROOT, "melody2d_b200", "csrc")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I" + csrc,
           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "emul", "error_stub.cpp"),
           os.path.join(csrc, "mel_material.cpp"), "-o", out]
    subprocess.run(cmd, check=True)
    L = C.CDLL(out)
    L.mel_update_matrices.restype = C.c_int
    L.emul_error.restype = C.c_char_p
    return L


def scene(material_type, flags):
    from test_oracle_laws import case_scene
    sc = case_scene("update_matrices")
    sc.update_matrices = (False,) + flags          # masses as loaded: the rebuilt ones run on the GPU path
    sc.materials = [(n, material_type if n == "Grain" else t, p) for (n, t, p) in sc.materials]
    return sc


@pytest.mark.parametrize("material_type", [0, 1])
@pytest.mark.parametrize("flags", [(True, True), (True, False), (False, True)])
def test_host_update_matches_oracle(matlib, oracle_built, material_type, flags):
    from melody2d_b200 import generator as g
    from melody2d_b200.abi import Desc
    from oracle.pyoracle import Oracle
    flat = g.flatten(scene(material_type, flags))
    n = len(flat["matrix_stiffness"])
    k0, c0 = np.array(flat["matrix_stiffness"], dtype=np.float64), np.array(flat["matrix_damping"], dtype=np.float64)
    k, c = k0.copy(), c0.copy()
    desc = Desc(flat)
    mass = np.ascontiguousarray(flat["node_mass"], dtype=np.float64)
    rc = matlib.mel_update_matrices(C.byref(desc.desc), mass.ctypes.data, k.ctypes.data, c.ctypes.data)
    assert rc == 0, matlib.emul_error()
    ko, co = Oracle(flat).matrices(n)
    np.testing.assert_array_equal(k, ko)
    np.testing.assert_array_equal(c, co)
    if flags[0]:
        assert not np.array_equal(k, k0)           # the file's matrices come from another modulus
        dofs = np.asarray(flat["matrix_dofs"]).reshape(-1, 2)
        assert np.all(k[dofs[:, 0] == dofs[:, 1]] > 0)   # the diagonal of an elastic stiffness
    else:
        np.testing.assert_array_equal(k, k0)
    if flags[1]:
        assert np.abs(c).max() > 0 and np.abs(c0).max() == 0
    else:
        np.testing.assert_array_equal(c, c0)
