"""Test infrastructure: Python handle on the C oracle (oracle/_build/libmeloracle.so).

Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from melody2d_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libmeloracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        vp = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(abi.MelModelDesc), C.POINTER(C.c_int), C.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_step.argtypes = [vp, C.c_int, C.c_int]
        L.orc_update_proximity.argtypes = [vp]
        L.orc_time.argtypes = [vp]; L.orc_time.restype = C.c_double
        L.orc_dt.argtypes = [vp]; L.orc_dt.restype = C.c_double
        L.orc_n_contacts.argtypes = [vp]
        L.orc_get_contacts.argtypes = [vp, C.POINTER(abi.MelContact), C.c_int]
        L.orc_set_contacts.argtypes = [vp, C.POINTER(abi.MelContact), C.c_int]
        for f in ("orc_get_node_state", "orc_set_node_state", "orc_get_positions", "orc_get_works", "orc_set_rigid", "orc_get_damage"):
            getattr(L, f).argtypes = [vp, C.POINTER(C.c_double)]
        L.orc_get_forces.argtypes = [vp] + [C.POINTER(C.c_double)] * 5
        L.orc_get_rigid.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_monitor.argtypes = [vp, C.POINTER(abi.MelMonitor)]
        L.orc_get_neighbours.argtypes = [vp, C.POINTER(C.c_int), C.c_int]
        L.orc_stale_shape_events.argtypes = [vp]; L.orc_stale_shape_events.restype = C.c_long
        L.orc_solver_stats.argtypes = [vp, C.POINTER(C.c_double)]
        L.orc_get_contact_pressures.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_set_time.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.orc_set_rsqrt_mode.argtypes = [C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_rsqrt_mode(correctly_rounded: bool) -> None:
    """0: x^(-1/2), cos and sin through glibc (pow, cos, sin) as the reference; 1: correctly rounded,
    as the GPU kernels."""
    lib().orc_set_rsqrt_mode(1 if correctly_rounded else 0)


class Oracle:
    """CPU restatement of the reference step on a flattened scene (generator.flatten)."""

    def __init__(self, flat: dict, n_regions: Optional[np.ndarray] = None, correctly_rounded: bool = False):
        self.L = lib()
        self.cr = bool(correctly_rounded)
        set_rsqrt_mode(self.cr)
        self.flat = flat
        self.desc = abi.Desc(flat)
        self.nn = len(flat["node_domain"])
        self.nb = len(flat["body_type"])
        h = C.c_void_p()
        regs = None
        if n_regions is not None:
            self._regs = np.ascontiguousarray(n_regions, dtype=np.int32)
            regs = self._regs.ctypes.data_as(C.POINTER(C.c_int))
        rc = self.L.orc_create(C.byref(self.desc.desc), regs, C.byref(h))
        if rc != 0:
            raise RuntimeError("orc_create failed")
        self.h = h

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int, proximity: bool = True):
        set_rsqrt_mode(self.cr)
        self.L.orc_step(self.h, int(n), 1 if proximity else 0)

    def update_proximity(self):
        set_rsqrt_mode(self.cr)
        self.L.orc_update_proximity(self.h)

    @property
    def time(self) -> float:
        return self.L.orc_time(self.h)

    @property
    def dt(self) -> float:
        return self.L.orc_dt(self.h)

    def node_state(self) -> np.ndarray:
        a = np.zeros(12 * self.nn)
        self.L.orc_get_node_state(self.h, _dp(a))
        return a.reshape(-1, 12)

    def set_node_state(self, st: np.ndarray):
        a = np.ascontiguousarray(st, dtype=np.float64).reshape(-1)
        self.L.orc_set_node_state(self.h, _dp(a))

    def body_status(self) -> np.ndarray:
        a = np.zeros(self.nb, dtype=np.int32)
        self.L.orc_get_body_status(self.h, a.ctypes.data_as(C.POINTER(C.c_int)))
        return a

    def update_damage(self, b: int) -> float:
        self.L.orc_update_damage.argtypes = [C.c_void_p, C.c_int]
        self.L.orc_update_damage.restype = C.c_double
        return self.L.orc_update_damage(self.h, int(b))

    def monitor_damage(self, bodies, cap: int = 10000):
        b = np.ascontiguousarray(bodies, dtype=np.int32)
        self.L.orc_monitor_damage.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_int]
        self.L.orc_monitor_damage(self.h, b.ctypes.data_as(C.POINTER(C.c_int)), len(b), int(cap))
        self._dmg = (len(b), cap)

    def damage_log(self) -> np.ndarray:
        n, cap = self._dmg
        out = np.zeros(cap * n)
        self.L.orc_damage_log.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        self.L.orc_damage_log.restype = C.c_int
        k = self.L.orc_damage_log(self.h, _dp(out))
        return out[: k * n].reshape(k, n)

    def damage(self) -> np.ndarray:
        a = np.zeros(self.nb)
        self.L.orc_get_damage(self.h, _dp(a))
        return a

    def matrices(self, n_matrix: int):
        """The MATRICES stiffness and damping entries as the set-up left them (after the updates
        of Body::Update_material)."""
        k, c = np.zeros(n_matrix), np.zeros(n_matrix)
        self.L.orc_get_matrices.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        self.L.orc_get_matrices.restype = C.c_int
        assert self.L.orc_get_matrices(self.h, _dp(k), _dp(c)) == n_matrix
        return k, c

    def positions(self) -> np.ndarray:
        a = np.zeros(2 * self.nn)
        self.L.orc_get_positions(self.h, _dp(a))
        return a.reshape(-1, 2)

    def forces(self):
        arrs = [np.zeros(2 * self.nn) for _ in range(5)]
        self.L.orc_get_forces(self.h, *[_dp(a) for a in arrs])
        return {k: a.reshape(-1, 2) for k, a in zip(("internal", "contact", "neumann", "dirichlet", "total"), arrs)}

    def rigid(self):
        r = np.zeros(abi.MEL_RIGID_NF * self.nb)
        f = np.zeros(12 * self.nb)
        self.L.orc_get_rigid(self.h, _dp(r), _dp(f))
        return r.reshape(self.nb, -1), f.reshape(self.nb, -1)

    def set_rigid(self, r: np.ndarray):
        a = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        self.L.orc_set_rigid(self.h, _dp(a))

    def works(self) -> np.ndarray:
        w = np.zeros(7 * self.nb)
        self.L.orc_get_works(self.h, _dp(w))
        return w.reshape(self.nb, 7)

    def contacts(self) -> np.ndarray:
        n = self.L.orc_n_contacts(self.h)
        buf = (abi.MelContact * max(1, n))()
        self.L.orc_get_contacts(self.h, buf, n)
        return abi.contacts_to_numpy(buf, n)

    def set_contacts(self, arr: np.ndarray):
        buf = abi.numpy_to_contacts(arr)
        if self.L.orc_set_contacts(self.h, buf, len(arr)) != 0:
            raise ValueError("bad contact list")

    def neighbours(self) -> np.ndarray:
        n = self.L.orc_get_neighbours(self.h, None, 0)
        rows = np.zeros(4 * max(1, n), dtype=np.int32)
        self.L.orc_get_neighbours(self.h, rows.ctypes.data_as(C.POINTER(C.c_int)), n)
        return rows[:4 * n].reshape(-1, 4)

    def monitor(self) -> abi.MelMonitor:
        m = abi.MelMonitor()
        self.L.orc_monitor(self.h, C.byref(m))
        return m

    def set_time(self, time: float, dt: float, next_contact_update: float):
        self.L.orc_set_time(self.h, float(time), float(dt), float(next_contact_update))

    def contact_pressures(self) -> np.ndarray:
        """(n_border_nodes, 2): x and y contact pressure of every border entry."""
        ne = int(np.asarray(self.flat["border_node_ptr"])[-1])
        px, py = np.zeros(max(ne, 1)), np.zeros(max(ne, 1))
        self.L.orc_get_contact_pressures(self.h, _dp(px), _dp(py))
        return np.stack([px[:ne], py[:ne]], axis=1)

    def stale_shape_events(self) -> int:
        return self.L.orc_stale_shape_events(self.h)

    def solver_stats(self) -> np.ndarray:
        a = np.zeros(5)
        self.L.orc_solver_stats(self.h, _dp(a))
        return a
