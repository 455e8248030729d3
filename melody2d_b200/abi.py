"""ctypes mirror of include/melgpu.h (structures and the library loader).

Field order follows the C declarations one for one; `make_desc` keeps the numpy arrays it points
at alive on the returned object."""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict

import numpy as np

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

MEL_RIGID_NF = 20
MEL_LAW_NPARAM = 11
MEL_MAT_NPARAM = 6
MEL_NINTERNAL = 3
MEL_DEACT_NF = 8

MEL_OK, MEL_ERR_INVALID, MEL_ERR_UNSUPPORTED, MEL_ERR_CUDA, MEL_ERR_OOM, MEL_ERR_NAN, MEL_ERR_BOUNDS, \
    MEL_ERR_TIMEOUT, MEL_ERR_IO, MEL_ERR_NO_DEVICE = range(10)
STATUS_NAMES = {0: "MEL_OK", 1: "MEL_ERR_INVALID", 2: "MEL_ERR_UNSUPPORTED", 3: "MEL_ERR_CUDA", 4: "MEL_ERR_OOM",
                5: "MEL_ERR_NAN", 6: "MEL_ERR_BOUNDS", 7: "MEL_ERR_TIMEOUT", 8: "MEL_ERR_IO", 9: "MEL_ERR_NO_DEVICE"}


class MelModelDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("period", C.c_double * 2), ("gravity", C.c_double * 2),
        ("time", C.c_double), ("dt", C.c_double), ("tend", C.c_double),
        ("contact_update_period", C.c_double), ("next_contact_update", C.c_double),
        ("solver", C.c_int), ("solver_params", C.c_double * 8), ("flags", C.c_int * 11),
        ("n_materials", C.c_int), ("material_type", _ip), ("material_params", _dp),
        ("n_laws", C.c_int), ("law_type", _ip), ("law_length", _ip), ("law_params", _dp), ("contacts_table", _ip),
        ("n_bodies", C.c_int), ("body_type", _ip), ("body_material", _ip), ("body_periodic", _ip), ("body_status", _ip),
        ("body_dist", _dp), ("body_node_ptr", _ip), ("body_border_ptr", _ip), ("body_gp_ptr", _ip), ("body_cell_ptr", _ip),
        ("rigid", _dp),
        ("n_nodes", C.c_int), ("node_x0", _dp), ("node_mass", _dp), ("node_inv_mass", _dp), ("node_domain", _dp),
        ("node_sup_ptr", _ip), ("node_sup_idx", _ip), ("node_sup_N", _dp), ("node_state", _dp),
        ("n_borders", C.c_int), ("border_body", _ip), ("border_periodicity", _ip), ("border_interpolant", _ip),
        ("border_before", _ip), ("border_after", _ip), ("border_node_ptr", _ip), ("border_nodes", _ip),
        ("border_bc_type", _ip), ("border_bc_param", _dp), ("border_hist_ptr", _ip), ("hist_time", _dp), ("hist_value", _dp),
        ("n_gauss", C.c_int), ("gp_sup_ptr", _ip), ("gp_sup_idx", _ip), ("gp_N", _dp), ("gp_dNdx", _dp), ("gp_dNdy", _dp),
        ("gp_weight", _dp), ("gp_jacobian", _dp),
        ("n_cells", C.c_int), ("cells", _ip),
        ("n_matrix", C.c_int), ("body_matrix_ptr", _ip), ("matrix_dofs", _ip), ("matrix_stiffness", _dp), ("matrix_damping", _dp),
        ("n_deactivated", C.c_int), ("deactivated", _dp),
        ("body_alid_ptr", _ip), ("alid_time", _dp), ("alid_value", _dp), ("node_alid", _dp),
    ]


class MelContact(C.Structure):
    _fields_ = [
        ("bodyS", C.c_int32), ("borderS", C.c_int32), ("border_nodeS", C.c_int32), ("nodeS", C.c_int32),
        ("bodyM", C.c_int32), ("borderM", C.c_int32), ("shiftM", C.c_int32), ("segmentM", C.c_int32),
        ("nodeM", C.c_int32 * 4), ("shiftMk", C.c_int32 * 4), ("shapeM", C.c_double * 4),
        ("gapn", C.c_double), ("vgapn", C.c_double), ("gapt", C.c_double), ("vgapt", C.c_double), ("xsi", C.c_double),
        ("xnorm", C.c_double), ("ynorm", C.c_double), ("xtan", C.c_double), ("ytan", C.c_double),
        ("effective_mass", C.c_double), ("length", C.c_double), ("fx", C.c_double), ("fy", C.c_double),
        ("nb_internal", C.c_int32), ("pad_", C.c_int32), ("internal", C.c_double * MEL_NINTERNAL),
    ]


class MelStepIO(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("run_proximity", C.c_int), ("time", C.c_double), ("dt", C.c_double),
                ("next_contact_update", C.c_double), ("n_contacts", C.c_int), ("n_proximity", C.c_int)]


class MelMonitor(C.Structure):
    _fields_ = [("time", C.c_double), ("kinetic_energy", C.c_double), ("mean_displacement", C.c_double * 2),
                ("rigid_force", C.c_double * 8), ("rigid_dirichlet", C.c_double * 8),
                ("active_contacts", C.c_int), ("n_contacts", C.c_int)]


MEL_MON_NF = 7
MEL_MON_MAX = 256
MEL_NFLAGS = 11


class MelSaveInfo(C.Structure):
    _fields_ = [("simulation_name", C.c_char_p), ("number_save", C.c_int), ("number_iteration", C.c_int),
                ("number_print", C.c_int), ("next_save", C.c_double), ("next_print", C.c_double)]


class MelRunControl(C.Structure):
    _fields_ = [("simulation_name", C.c_char * 256), ("save_period", C.c_double), ("print_period", C.c_double),
                ("next_save", C.c_double), ("next_print", C.c_double), ("number_save", C.c_int),
                ("number_iteration", C.c_int), ("number_print", C.c_int), ("n_monitored", C.c_int),
                ("monitored", C.c_double * (MEL_MON_MAX * MEL_MON_NF)), ("flags", C.c_int * MEL_NFLAGS)]


class MelOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("use_graph", C.c_int), ("max_contacts", C.c_int)]


# numpy structured dtype with the same layout as mel_contact (for bulk transfers)
CONTACT_DTYPE = np.dtype([
    ("bodyS", "<i4"), ("borderS", "<i4"), ("border_nodeS", "<i4"), ("nodeS", "<i4"),
    ("bodyM", "<i4"), ("borderM", "<i4"), ("shiftM", "<i4"), ("segmentM", "<i4"),
    ("nodeM", "<i4", 4), ("shiftMk", "<i4", 4), ("shapeM", "<f8", 4),
    ("gapn", "<f8"), ("vgapn", "<f8"), ("gapt", "<f8"), ("vgapt", "<f8"), ("xsi", "<f8"),
    ("xnorm", "<f8"), ("ynorm", "<f8"), ("xtan", "<f8"), ("ytan", "<f8"),
    ("effective_mass", "<f8"), ("length", "<f8"), ("fx", "<f8"), ("fy", "<f8"),
    ("nb_internal", "<i4"), ("pad_", "<i4"), ("internal", "<f8", MEL_NINTERNAL)])
assert CONTACT_DTYPE.itemsize == C.sizeof(MelContact)


class Desc:
    """A filled MelModelDesc plus the arrays it references."""

    def __init__(self, flat: Dict):
        self.arrays = {}
        d = MelModelDesc()
        d.abi_version = 2

        def dptr(name):
            a = np.ascontiguousarray(np.asarray(flat[name], dtype=np.float64))
            self.arrays[name] = a
            return a.ctypes.data_as(_dp)

        def iptr(name):
            a = np.ascontiguousarray(np.asarray(flat[name], dtype=np.int32))
            self.arrays[name] = a
            return a.ctypes.data_as(_ip)

        d.period[:] = list(flat["period"])
        d.gravity[:] = list(flat["gravity"])
        d.time = float(flat["time"]); d.dt = float(flat["dt"]); d.tend = float(flat["tend"])
        d.contact_update_period = float(flat["contact_update_period"])
        d.next_contact_update = float(flat["next_contact_update"])
        d.solver = int(flat["solver"])
        d.solver_params[:] = [float(x) for x in flat["solver_params"]]
        d.flags[:] = [int(x) for x in flat["flags"]]
        d.n_materials = len(flat["material_type"])
        d.material_type = iptr("material_type"); d.material_params = dptr("material_params")
        d.n_laws = len(flat["law_type"])
        d.law_type = iptr("law_type"); d.law_length = iptr("law_length"); d.law_params = dptr("law_params")
        d.contacts_table = iptr("contacts_table")
        d.n_bodies = len(flat["body_type"])
        for k in ("body_type", "body_material", "body_periodic", "body_status", "body_node_ptr", "body_border_ptr",
                  "body_gp_ptr", "body_cell_ptr"):
            setattr(d, k, iptr(k))
        d.body_dist = dptr("body_dist"); d.rigid = dptr("rigid")
        d.n_nodes = len(flat["node_domain"])
        for k in ("node_x0", "node_mass", "node_inv_mass", "node_domain", "node_sup_N", "node_state"):
            setattr(d, k, dptr(k))
        d.node_sup_ptr = iptr("node_sup_ptr"); d.node_sup_idx = iptr("node_sup_idx")
        d.n_borders = len(flat["border_body"])
        for k in ("border_body", "border_periodicity", "border_interpolant", "border_before", "border_after",
                  "border_node_ptr", "border_nodes", "border_bc_type", "border_hist_ptr"):
            setattr(d, k, iptr(k))
        d.border_bc_param = dptr("border_bc_param"); d.hist_time = dptr("hist_time"); d.hist_value = dptr("hist_value")
        d.n_gauss = len(flat["gp_weight"])
        d.gp_sup_ptr = iptr("gp_sup_ptr"); d.gp_sup_idx = iptr("gp_sup_idx")
        for k in ("gp_N", "gp_dNdx", "gp_dNdy", "gp_weight", "gp_jacobian"):
            setattr(d, k, dptr(k))
        d.n_cells = len(flat["cells"]) // 3
        d.cells = iptr("cells")
        d.n_matrix = len(flat["matrix_stiffness"])
        d.body_matrix_ptr = iptr("body_matrix_ptr"); d.matrix_dofs = iptr("matrix_dofs")
        d.matrix_stiffness = dptr("matrix_stiffness"); d.matrix_damping = dptr("matrix_damping")
        deact = np.asarray(flat.get("deactivated", np.zeros((0, MEL_DEACT_NF))), dtype=np.float64).reshape(-1, MEL_DEACT_NF)
        d.n_deactivated = deact.shape[0]
        if deact.shape[0]:
            self.arrays["deactivated"] = np.ascontiguousarray(deact.reshape(-1))
            d.deactivated = self.arrays["deactivated"].ctypes.data_as(_dp)
        if "body_alid_ptr" in flat and len(flat["alid_time"]) > 0:      # ALID layers
            d.body_alid_ptr = iptr("body_alid_ptr")
            d.alid_time = dptr("alid_time"); d.alid_value = dptr("alid_value"); d.node_alid = dptr("node_alid")
        self.desc = d

    def ref(self):
        return C.byref(self.desc)


def contacts_to_numpy(buf, n: int) -> np.ndarray:
    arr = np.frombuffer((C.c_char * (n * CONTACT_DTYPE.itemsize)).from_address(C.addressof(buf)), dtype=CONTACT_DTYPE)
    return arr.copy()


def numpy_to_contacts(arr: np.ndarray):
    arr = np.ascontiguousarray(arr, dtype=CONTACT_DTYPE)
    buf = (MelContact * max(1, len(arr)))()
    C.memmove(buf, arr.ctypes.data, arr.nbytes)
    return buf
