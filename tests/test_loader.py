"""The library's reader of STATIC_CONTROL / STATIC_DATA / DYNAMIC files reproduces the flattened
model the generator wrote (Load_static / Load_dynamic token order, Code/IO.h:598-2345)."""
import numpy as np

from conftest import flat_of, squeezed_lattice


def test_asc_roundtrip(tmp_path, gpu_lib):
    from melody2d_b200 import generator as g, solver
    scene = squeezed_lattice(3, 3)
    g.write_asc(scene, str(tmp_path))
    d = solver.load_desc_arrays(str(tmp_path))
    f = flat_of(scene)
    for k, v in f.items():
        if k == "material_names":
            continue
        np.testing.assert_array_equal(np.asarray(v), np.asarray(d[k]), err_msg=k)


def test_missing_files_report_io_error(tmp_path, gpu_lib):
    from melody2d_b200 import solver
    import pytest
    with pytest.raises(solver.MelError) as e:
        solver.load_desc_arrays(str(tmp_path / "nope"))
    assert e.value.code == 8


def test_asc_roundtrip_matrices_deactivation_alid(tmp_path, gpu_lib):
    """MATRICES (Code/IO.h:1827-1851) and DEACTIVATION entries (Read_spy_line plus below / equal /
    above and the threshold, Code/IO.h:947-968) read back as the generator encoded them, and so do
    the UPDATE_MASS/STIFFNESS/DAMPING_MATRIX lines of DYNAMIC (flags[4..6], Code/IO.h:1920-1925)."""
    import sys, os
    sys.path.insert(0, os.path.dirname(__file__))
    from melody2d_b200 import generator as g, solver
    from test_oracle_laws import case_scene
    for name in ("damping", "deactivation", "alid", "update_matrices"):
        scene = case_scene(name)
        d_ = tmp_path / name
        g.write_asc(scene, str(d_))
        d = solver.load_desc_arrays(str(d_))
        f = g.flatten(scene)
        keys = ["body_matrix_ptr", "matrix_dofs", "matrix_stiffness", "matrix_damping", "deactivated", "flags"]
        if name == "update_matrices":
            assert list(np.asarray(d["flags"])[4:7]) == [1, 1, 1]
        if name in ("alid", "update_matrices"):
            # the ALID block (Code/IO.h:1395-1480) and the nodal coefficients the loader computes
            # from the initial positions (Code/IO.h:1548-1600), equal to the generator's
            keys += ["body_alid_ptr", "alid_time", "alid_value", "node_alid"]
            assert np.count_nonzero(f["node_alid"]) > 0
        for k in keys:
            np.testing.assert_array_equal(np.asarray(f[k]), np.asarray(d[k]), err_msg=(name, k))
