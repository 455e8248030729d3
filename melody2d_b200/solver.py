"""Python mirror of the solver's C ABI (include/melgpu.h) over libmelgpu.so.

    s = Solver.from_flat(generator.flatten(scene))      # or Solver.from_files(dir)
    s.step(100)                                          # Euler_step + proximity cadence
    st = s.node_state()                                  # u, v, a, up, vp, ap per node

The library is required: importing works without it, but every constructor raises if
libmelgpu.so cannot be loaded or no CUDA device is present (there is no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmelgpu.so")
_lib = None

# every exported entry point with its argument types (restype is mel_status unless stated)
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
SIGNATURES = {
    "mel_create": [C.POINTER(abi.MelModelDesc), C.POINTER(abi.MelOptions), C.POINTER(_vp)],
    "mel_create_from_files": [C.c_char_p, C.c_int, C.POINTER(abi.MelOptions), C.POINTER(_vp)],
    "mel_destroy": [_vp],
    "mel_step": [_vp, C.POINTER(abi.MelStepIO)],
    "mel_update_proximity": [_vp],
    "mel_set_contacts": [_vp, C.POINTER(abi.MelContact), C.c_int],
    "mel_get_node_state": [_vp, _dp],
    "mel_set_node_state": [_vp, _dp],
    "mel_pin_host": [_vp, C.c_size_t],
    "mel_unpin_host": [_vp],
    "mel_get_positions": [_vp, _dp],
    "mel_get_forces": [_vp, _dp, _dp, _dp, _dp, _dp],
    "mel_get_rigid": [_vp, _dp, _dp],
    "mel_get_works": [_vp, _dp],
    "mel_get_contact_count": [_vp, _ip],
    "mel_get_contact_pressures": [_vp, _dp, _dp],
    "mel_get_solver_stats": [_vp, _dp],
    "mel_get_contacts": [_vp, C.POINTER(abi.MelContact), C.c_int, _ip],
    "mel_get_time": [_vp, _dp, _dp],
    "mel_checkpoint_start": [_vp],
    "mel_checkpoint_read": [_vp, _dp, _dp, _dp, C.POINTER(abi.MelContact), C.c_int, _ip, _dp],
    "mel_monitor_compute": [_vp, C.POINTER(abi.MelMonitor)],
    "mel_set_rigid": [_vp, _dp],
    "mel_set_time": [_vp, C.c_double, C.c_double, C.c_double],
    "mel_record_forces": [_vp, C.c_int],
    "mel_set_timing": [_vp, C.c_int],
    "mel_get_error_words": [_vp, C.POINTER(C.c_uint), C.c_int],
    "mel_load_desc": [C.c_char_p, C.c_int, C.POINTER(C.POINTER(abi.MelModelDesc)), C.POINTER(_vp)],
    "mel_free_desc": [_vp],
    "mel_get_kernel_times": [_vp, _dp, _dp, _dp, _dp, _ip],
    "mel_get_sizes": [_vp, _ip, _ip, _ip, _ip, _ip, _ip],
    "mel_get_step_stats": [_vp, _dp, _dp, _dp, _ip, _ip],
    "mel_monitor_reduce_static": [_vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp],
    "mel_batch_create": [C.c_int, C.c_int, C.POINTER(_vp)],
    "mel_batch_admit": [_vp, _vp],
    "mel_batch_retire": [_vp, _vp],
    "mel_batch_step": [_vp, C.c_int, C.c_int],
    "mel_batch_stats": [_vp, _dp, C.POINTER(C.c_longlong), _ip],
    "mel_batch_destroy": [_vp],
    "mel_get_health": [_vp, _ip],
    "mel_get_bc_pressures": [_vp, _dp, _dp],
    "mel_get_body_status": [_vp, _ip],
    "mel_get_kernel_config": [_vp, _ip, C.POINTER(C.c_longlong), _ip],
    "mel_monitor_setup": [_vp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _ip],
    "mel_monitor_rows": [_vp, _dp, C.c_int, _ip],
    "mel_write_dynamic": [_vp, C.c_char_p, C.POINTER(abi.MelSaveInfo)],
    "mel_load_run_control": [_vp, C.POINTER(abi.MelRunControl)],
    "mel_create_loaded": [_vp, C.POINTER(abi.MelOptions), C.POINTER(_vp)],
    "mel_mls_shapes": [C.c_int, _ip, _dp, _dp, _ip, _dp, C.POINTER(C.c_longlong), _ip, _dp, _dp, _dp,
                       C.c_longlong, C.POINTER(C.c_longlong), C.c_int, _dp],
}


class PinnedArray:
    """A float64 numpy array page-locked with mel_pin_host for fast state transfers (released by
    close())."""

    def __init__(self, shape):
        self.array = np.zeros(shape, dtype=np.float64)
        _check(lib().mel_pin_host(self.array.ctypes.data, self.array.nbytes))
        self._pinned = True

    def close(self):
        if self._pinned:
            lib().mel_unpin_host(self.array.ctypes.data)
            self._pinned = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads libmelgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m melody2d_b200.build`")
        # the chunk-size tuning table written by melody2d_b200.autotune, unless the caller names one
        table = os.path.join(_HERE, "tuning.txt")
        if "MELGPU_TUNE_FILE" not in os.environ and os.path.exists(table):
            os.environ["MELGPU_TUNE_FILE"] = table
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.mel_last_error_string.restype = C.c_char_p
        L.mel_last_error_string.argtypes = []
        L.mel_abi_version.restype = C.c_int
        L.mel_abi_version.argtypes = []
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise MelError(rc, lib().mel_last_error_string().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Solver:
    """One resident model on one GPU (a mel_handle)."""

    def __init__(self, handle, nn: int, nb: int, keep=None):
        self.h = handle
        self.nn = nn
        self.nb = nb
        self._keep = keep
        self._mon_len = 0

    # ---- construction -------------------------------------------------------------------
    @classmethod
    def from_flat(cls, flat: dict, precision: int = 0, device: int = 0, retain: bool = True) -> "Solver":
        """retain=False drops the references to the description's arrays once mel_create has
        returned (the handle keeps its own copies), so that arrays mapped from shared memory can
        be released while the solver lives."""
        L = lib()
        desc = abi.Desc(flat)
        opt = abi.MelOptions(precision=precision, device=device, use_graph=0, max_contacts=0)
        h = C.c_void_p()
        _check(L.mel_create(C.byref(desc.desc), C.byref(opt), C.byref(h)))
        return cls(h, len(flat["node_domain"]), len(flat["body_type"]), keep=desc if retain else None)

    @classmethod
    def from_files(cls, directory: str, restart_index: int = 0, precision: int = 0, device: int = 0) -> "Solver":
        L = lib()
        opt = abi.MelOptions(precision=precision, device=device, use_graph=0, max_contacts=0)
        h = C.c_void_p()
        _check(L.mel_create_from_files(directory.encode(), restart_index, C.byref(opt), C.byref(h)))
        s = cls(h, 0, 0)
        sizes = s.sizes()
        s.nn, s.nb = sizes["n_nodes"], sizes["n_bodies"]
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().mel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- stepping -------------------------------------------------------------------------
    def step(self, n: int = 1, proximity: bool = True) -> abi.MelStepIO:
        io = abi.MelStepIO(nsteps=int(n), run_proximity=1 if proximity else 0)
        _check(lib().mel_step(self.h, C.byref(io)))
        return io

    def update_proximity(self):
        _check(lib().mel_update_proximity(self.h))

    # ---- state ----------------------------------------------------------------------------
    def node_state(self) -> np.ndarray:
        a = np.zeros(12 * self.nn)
        _check(lib().mel_get_node_state(self.h, _ptr(a)))
        return a.reshape(-1, 12)

    def set_node_state(self, st: np.ndarray):
        a = np.ascontiguousarray(st, dtype=np.float64).reshape(-1)
        _check(lib().mel_set_node_state(self.h, _ptr(a)))

    def positions(self) -> np.ndarray:
        a = np.zeros(2 * self.nn)
        _check(lib().mel_get_positions(self.h, _ptr(a)))
        return a.reshape(-1, 2)

    def record_forces(self, on: bool = True):
        _check(lib().mel_record_forces(self.h, 1 if on else 0))

    def set_timing(self, on: bool = True):
        _check(lib().mel_set_timing(self.h, 1 if on else 0))

    def forces(self) -> dict:
        arrs = [np.zeros(2 * self.nn) for _ in range(5)]
        _check(lib().mel_get_forces(self.h, *[_ptr(a) for a in arrs]))
        return {k: a.reshape(-1, 2) for k, a in zip(("internal", "contact", "neumann", "dirichlet", "total"), arrs)}

    def rigid(self):
        r = np.zeros(abi.MEL_RIGID_NF * self.nb)
        f = np.zeros(12 * self.nb)
        _check(lib().mel_get_rigid(self.h, _ptr(r), _ptr(f)))
        return r.reshape(self.nb, -1), f.reshape(self.nb, -1)

    def set_rigid(self, r: np.ndarray):
        a = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        _check(lib().mel_set_rigid(self.h, _ptr(a)))

    def set_time(self, time: float, dt: float, next_contact_update: float):
        _check(lib().mel_set_time(self.h, float(time), float(dt), float(next_contact_update)))

    def works(self) -> np.ndarray:
        w = np.zeros(7 * self.nb)
        _check(lib().mel_get_works(self.h, _ptr(w)))
        return w.reshape(self.nb, 7)

    def contacts(self) -> np.ndarray:
        n = C.c_int()
        _check(lib().mel_get_contact_count(self.h, C.byref(n)))
        buf = (abi.MelContact * max(1, n.value))()
        _check(lib().mel_get_contacts(self.h, buf, n.value, C.byref(n)))
        return abi.contacts_to_numpy(buf, n.value)

    def solver_stats(self) -> np.ndarray:
        """Solver_step statistics of the last accepted step: neval, max_error, mean_error, total_mass,
        max_mass."""
        a = np.zeros(5)
        _check(lib().mel_get_solver_stats(self.h, _ptr(a)))
        return a

    def contact_pressures(self) -> np.ndarray:
        """(n_border_nodes, 2): x and y contact pressure of every border entry after the last step."""
        ne = self.sizes()["n_border_nodes"]
        px, py = np.zeros(max(ne, 1)), np.zeros(max(ne, 1))
        _check(lib().mel_get_contact_pressures(self.h, _ptr(px), _ptr(py)))
        return np.stack([px[:ne], py[:ne]], axis=1)

    def body_status(self) -> np.ndarray:
        """MEL_STATUS_* of every body (Update_status can turn bodies inactive)."""
        a = np.zeros(self.nb, dtype=np.int32)
        _check(lib().mel_get_body_status(self.h, a.ctypes.data_as(_ip)))
        return a

    def bc_pressures(self) -> np.ndarray:
        """Border-condition pressures of the last step, (n_border_entries, 2)."""
        ne = self.sizes()["n_border_nodes"]
        px = np.zeros(max(ne, 1)); py = np.zeros(max(ne, 1))
        _check(lib().mel_get_bc_pressures(self.h, _ptr(px), _ptr(py)))
        return np.stack([px[:ne], py[:ne]], axis=1)

    def monitor_setup(self, monitored, energy: bool = False, boundaries: bool = False, ring_rows: int = 1000,
                      first_iteration: int = 0) -> int:
        """Device Monitoring (mel_monitor_setup): `monitored` is a list of Read_spy_line vectors;
        returns the longest row."""
        m = np.zeros((max(len(monitored), 1), abi.MEL_MON_NF))
        for i, e in enumerate(monitored):
            m[i, :len(e)] = e
        L = C.c_int()
        _check(lib().mel_monitor_setup(self.h, _ptr(m), len(monitored), int(energy), int(boundaries), ring_rows,
                                       first_iteration, C.byref(L)))
        self._mon_len = L.value
        return L.value

    def monitor_rows(self) -> list:
        """The monitoring rows recorded since the last call, one float64 array each."""
        n = C.c_int()
        _check(lib().mel_monitor_rows(self.h, None, 0, C.byref(n)))
        if n.value == 0:
            return []
        stride = self._mon_len + 1
        buf = np.zeros(n.value * stride)
        _check(lib().mel_monitor_rows(self.h, _ptr(buf), n.value, C.byref(n)))
        rows = buf.reshape(n.value, stride)
        return [r[1:1 + int(r[0])].copy() for r in rows]

    def write_dynamic(self, directory: str, number_save: int, number_iteration: int, number_print: int = 0,
                      next_save: float = 0.0, next_print: float = 0.0, name: str = "") -> str:
        """Write_dynamic: <directory>/DYNAMIC_<number_save>.asc in the reference's layout."""
        info = abi.MelSaveInfo(name.encode(), number_save, number_iteration, number_print, next_save, next_print)
        _check(lib().mel_write_dynamic(self.h, directory.encode(), C.byref(info)))
        return os.path.join(directory, "DYNAMIC_%05d.asc" % number_save)

    def set_contacts(self, arr: np.ndarray):
        buf = abi.numpy_to_contacts(arr)
        _check(lib().mel_set_contacts(self.h, buf, len(arr)))

    def health(self):
        """(0, "") for a healthy solver, else (status, message) of the failure that retired it
        from its batch."""
        f = C.c_int()
        _check(lib().mel_get_health(self.h, C.byref(f)))
        return f.value, (lib().mel_last_error_string().decode(errors="replace") if f.value else "")

    def checkpoint_start(self):
        """Snapshot of the state, copied to host memory while later steps run (mel_checkpoint_start)."""
        _check(lib().mel_checkpoint_start(self.h))

    def checkpoint_read(self) -> dict:
        """The snapshot of the last checkpoint_start: node_state (n_nodes, 12), rigid, works
        (n_bodies, 7), contacts (as contacts()), time, dt, next_contact_update."""
        n = C.c_int()
        t3 = np.zeros(3)
        st = np.zeros(12 * self.nn)
        rg = np.zeros(abi.MEL_RIGID_NF * self.nb)
        wk = np.zeros(7 * self.nb)
        cap = self.contact_capacity_hint()
        while True:
            buf = (abi.MelContact * max(1, cap))()
            rc = lib().mel_checkpoint_read(self.h, _ptr(st), _ptr(rg), _ptr(wk), buf, cap, C.byref(n), _ptr(t3))
            if rc == 0:
                break
            if n.value > cap:              # buffer too small: the snapshot stays pending, retry
                cap = n.value
                continue
            _check(rc)
        return {"node_state": st.reshape(-1, 12), "rigid": rg.reshape(self.nb, -1), "works": wk.reshape(self.nb, 7),
                "contacts": abi.contacts_to_numpy(buf, n.value), "time": t3[0], "dt": t3[1],
                "next_contact_update": t3[2]}

    def contact_capacity_hint(self) -> int:
        n = C.c_int()
        _check(lib().mel_get_contact_count(self.h, C.byref(n)))
        return max(16, 2 * n.value)

    def time(self):
        t = C.c_double(); dt = C.c_double()
        _check(lib().mel_get_time(self.h, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def monitor(self) -> abi.MelMonitor:
        m = abi.MelMonitor()
        _check(lib().mel_monitor_compute(self.h, C.byref(m)))
        return m

    def error_words(self) -> np.ndarray:
        w = (C.c_uint * 9)()
        _check(lib().mel_get_error_words(self.h, w, 9))
        return np.array(list(w), dtype=np.uint32)

    def kernel_times(self) -> dict:
        v = [C.c_double() for _ in range(4)]
        n = C.c_int()
        _check(lib().mel_get_kernel_times(self.h, *[C.byref(x) for x in v], C.byref(n)))
        return dict(contact=v[0].value, body=v[1].value, rigid=v[2].value, proximity=v[3].value, launches=n.value)

    def step_stats(self) -> dict:
        v = [C.c_double() for _ in range(3)]
        n = [C.c_int() for _ in range(2)]
        _check(lib().mel_get_step_stats(self.h, *[C.byref(x) for x in v], *[C.byref(x) for x in n]))
        return dict(ms_total=v[0].value, bytes_body=v[1].value, bytes_contact=v[2].value,
                    n_deformable_nodes=n[0].value, n_contacts=n[1].value)

    def kernel_config(self) -> dict:
        """Body-kernel launch configuration: chunk entry cap, shared memory per CTA, CTAs."""
        cap, ctas = C.c_int(), C.c_int()
        smem = C.c_longlong()
        _check(lib().mel_get_kernel_config(self.h, C.byref(cap), C.byref(smem), C.byref(ctas)))
        return {"chunk_cap": cap.value, "body_smem": smem.value, "body_ctas": ctas.value}

    def sizes(self) -> dict:
        v = [C.c_int() for _ in range(6)]
        _check(lib().mel_get_sizes(self.h, *[C.byref(x) for x in v]))
        keys = ("n_bodies", "n_nodes", "n_gauss", "n_gp_entries", "n_node_entries", "n_border_nodes")
        return {k: x.value for k, x in zip(keys, v)}


def mls_shapes(bodies, device: int = 0, timing: Optional[dict] = None):
    """Shape functions at Gauss points on the device (mel_mls_shapes) for a list of bodies, each a
    (points (P,2), nodes (n,2), radii (n,)) triple.  Returns one (ptr, idx, N, dNdx, dNdy) CSR
    tuple per body, the layout generator.mls_shape returns.  `timing`, when given, receives the
    value pass's device milliseconds."""
    bnp = np.zeros(len(bodies) + 1, dtype=np.int32)
    bpp = np.zeros(len(bodies) + 1, dtype=np.int32)
    for i, (pts, nodes, radii) in enumerate(bodies):
        bnp[i + 1] = bnp[i] + nodes.shape[0]
        bpp[i + 1] = bpp[i] + pts.shape[0]
    nodes = np.ascontiguousarray(np.concatenate([b[1] for b in bodies]), dtype=np.float64)
    radii = np.ascontiguousarray(np.concatenate([b[2] for b in bodies]), dtype=np.float64)
    pts = np.ascontiguousarray(np.concatenate([b[0] for b in bodies]), dtype=np.float64)
    np_ = int(bpp[-1])
    ptr = np.zeros(np_ + 1, dtype=np.int64)
    ne = C.c_longlong()
    ip = lambda a: a.ctypes.data_as(_ip)
    lp = ptr.ctypes.data_as(C.POINTER(C.c_longlong))
    L = lib()
    _check(L.mel_mls_shapes(len(bodies), ip(bnp), _ptr(nodes), _ptr(radii), ip(bpp), _ptr(pts), lp, None, None,
                            None, None, 0, C.byref(ne), device, None))
    n = ne.value
    idx = np.zeros(max(n, 1), dtype=np.int32)
    N, Nx, Ny = np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1))
    ms = C.c_double()
    _check(L.mel_mls_shapes(len(bodies), ip(bnp), _ptr(nodes), _ptr(radii), ip(bpp), _ptr(pts), lp, ip(idx),
                            _ptr(N), _ptr(Nx), _ptr(Ny), n, C.byref(ne), device, C.byref(ms)))
    if timing is not None:
        timing["kernel_ms"] = ms.value
    out = []
    for i in range(len(bodies)):
        a, b = int(bpp[i]), int(bpp[i + 1])
        e0, e1 = int(ptr[a]), int(ptr[b])
        out.append((ptr[a:b + 1] - e0, idx[e0:e1].astype(np.int64), N[e0:e1], Nx[e0:e1], Ny[e0:e1]))
    return out


def load_run_control(directory: str, restart_index: int = 0) -> dict:
    """What the input files say about output (mel_load_run_control): periods, counters, the
    MONITORING entries (Read_spy_line vectors) and the DYNAMIC flags.  No GPU needed."""
    L = lib()
    dp = C.POINTER(abi.MelModelDesc)()
    owner = C.c_void_p()
    _check(L.mel_load_desc(directory.encode(), restart_index, C.byref(dp), C.byref(owner)))
    try:
        rc = abi.MelRunControl()
        _check(L.mel_load_run_control(owner, C.byref(rc)))
        mon = np.ctypeslib.as_array(rc.monitored).reshape(abi.MEL_MON_MAX, abi.MEL_MON_NF)[:rc.n_monitored].copy()
        return {"simulation_name": rc.simulation_name.decode(), "save_period": rc.save_period,
                "print_period": rc.print_period, "next_save": rc.next_save, "next_print": rc.next_print,
                "number_save": rc.number_save, "number_iteration": rc.number_iteration,
                "number_print": rc.number_print, "monitored": mon, "flags": list(rc.flags)}
    finally:
        L.mel_free_desc(owner)


def load_desc_arrays(directory: str, restart_index: int = 0) -> dict:
    """Parses the reference's input files with the library's loader (no GPU needed) and returns
    the flattened arrays (same keys as generator.flatten)."""
    L = lib()
    dp = C.POINTER(abi.MelModelDesc)()
    owner = C.c_void_p()
    _check(L.mel_load_desc(directory.encode(), restart_index, C.byref(dp), C.byref(owner)))
    try:
        d = dp.contents
        out = {}
        def arr(ptr, n, dtype):
            if n <= 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy()
        nb, nn, nbd, ng, nm = d.n_bodies, d.n_nodes, d.n_borders, d.n_gauss, d.n_materials
        out["period"] = np.array(list(d.period)); out["gravity"] = np.array(list(d.gravity))
        out["time"] = d.time; out["dt"] = d.dt; out["tend"] = d.tend
        out["contact_update_period"] = d.contact_update_period; out["next_contact_update"] = d.next_contact_update
        out["solver"] = d.solver; out["solver_params"] = np.array(list(d.solver_params)); out["flags"] = np.array(list(d.flags))
        out["material_type"] = arr(d.material_type, nm, np.int32)
        out["material_params"] = arr(d.material_params, nm * abi.MEL_MAT_NPARAM, np.float64)
        out["law_type"] = arr(d.law_type, d.n_laws, np.int32); out["law_length"] = arr(d.law_length, d.n_laws, np.int32)
        out["law_params"] = arr(d.law_params, d.n_laws * abi.MEL_LAW_NPARAM, np.float64)
        out["contacts_table"] = arr(d.contacts_table, nm * nm, np.int32)
        for k in ("body_type", "body_material", "body_periodic", "body_status"):
            out[k] = arr(getattr(d, k), nb, np.int32)
        out["body_dist"] = arr(d.body_dist, 3 * nb, np.float64)
        for k in ("body_node_ptr", "body_border_ptr", "body_gp_ptr", "body_cell_ptr"):
            out[k] = arr(getattr(d, k), nb + 1, np.int32)
        out["rigid"] = arr(d.rigid, nb * abi.MEL_RIGID_NF, np.float64)
        out["node_x0"] = arr(d.node_x0, 2 * nn, np.float64); out["node_mass"] = arr(d.node_mass, 2 * nn, np.float64)
        out["node_inv_mass"] = arr(d.node_inv_mass, 2 * nn, np.float64); out["node_domain"] = arr(d.node_domain, nn, np.float64)
        out["node_sup_ptr"] = arr(d.node_sup_ptr, nn + 1, np.int32)
        ns = int(out["node_sup_ptr"][-1])
        out["node_sup_idx"] = arr(d.node_sup_idx, ns, np.int32); out["node_sup_N"] = arr(d.node_sup_N, ns, np.float64)
        out["node_state"] = arr(d.node_state, 12 * nn, np.float64)
        for k in ("border_body", "border_periodicity", "border_interpolant", "border_before", "border_after"):
            out[k] = arr(getattr(d, k), nbd, np.int32)
        out["border_node_ptr"] = arr(d.border_node_ptr, nbd + 1, np.int32)
        ne = int(out["border_node_ptr"][-1])
        out["border_nodes"] = arr(d.border_nodes, ne, np.int32)
        out["border_bc_type"] = arr(d.border_bc_type, 2 * nbd, np.int32)
        out["border_bc_param"] = arr(d.border_bc_param, 4 * nbd, np.float64)
        out["border_hist_ptr"] = arr(d.border_hist_ptr, 2 * nbd + 1, np.int32)
        nh = int(out["border_hist_ptr"][-1])
        out["hist_time"] = arr(d.hist_time, nh, np.float64); out["hist_value"] = arr(d.hist_value, nh, np.float64)
        out["gp_sup_ptr"] = arr(d.gp_sup_ptr, ng + 1, np.int32)
        nge = int(out["gp_sup_ptr"][-1])
        out["gp_sup_idx"] = arr(d.gp_sup_idx, nge, np.int32)
        for k in ("gp_N", "gp_dNdx", "gp_dNdy"):
            out[k] = arr(getattr(d, k), nge, np.float64)
        out["gp_weight"] = arr(d.gp_weight, ng, np.float64); out["gp_jacobian"] = arr(d.gp_jacobian, ng, np.float64)
        out["cells"] = arr(d.cells, 3 * d.n_cells, np.int32)
        out["body_matrix_ptr"] = arr(d.body_matrix_ptr, nb + 1, np.int32)
        out["matrix_dofs"] = arr(d.matrix_dofs, 2 * d.n_matrix, np.int32)
        out["matrix_stiffness"] = arr(d.matrix_stiffness, d.n_matrix, np.float64)
        out["matrix_damping"] = arr(d.matrix_damping, d.n_matrix, np.float64)
        out["deactivated"] = arr(d.deactivated, d.n_deactivated * abi.MEL_DEACT_NF, np.float64).reshape(-1, abi.MEL_DEACT_NF)
        if d.body_alid_ptr:
            out["body_alid_ptr"] = arr(d.body_alid_ptr, 2 * nb + 1, np.int32)
            na = int(out["body_alid_ptr"][-1])
            out["alid_time"] = arr(d.alid_time, na, np.float64); out["alid_value"] = arr(d.alid_value, na, np.float64)
            out["node_alid"] = arr(d.node_alid, 2 * nn, np.float64)
        return out
    finally:
        L.mel_free_desc(owner)


class Batch:
    """Several independent solvers advanced by shared launches (mel_batch_*): admit handles,
    step them together, retire them when their run ends.  Each member's results are those it
    would have on its own."""

    def __init__(self, precision: int = 0, device: int = 0):
        self.b = C.c_void_p()
        _check(lib().mel_batch_create(int(device), int(precision), C.byref(self.b)))
        self.members = []

    def admit(self, s: Solver):
        _check(lib().mel_batch_admit(self.b, s.h))
        self.members.append(s)

    def retire(self, s: Solver):
        _check(lib().mel_batch_retire(self.b, s.h))
        self.members.remove(s)

    def step(self, n: int = 1, proximity: bool = True) -> list:
        """Advances every member; returns the members that diverged during the call (they have
        left the batch; `Solver.health()` gives the reason)."""
        _check(lib().mel_batch_step(self.b, int(n), 1 if proximity else 0))
        failed = [s for s in self.members if s.health()[0]]
        for s in failed:
            self.members.remove(s)
        return failed

    def stats(self) -> dict:
        ms, launches, members = C.c_double(), C.c_longlong(), C.c_int()
        _check(lib().mel_batch_stats(self.b, C.byref(ms), C.byref(launches), C.byref(members)))
        return {"ms_last_call": ms.value, "launches": launches.value, "members": members.value}

    def close(self):
        if getattr(self, "b", None):
            lib().mel_batch_destroy(self.b)
            self.b = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
