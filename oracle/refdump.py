"""Test infrastructure: reader for the binary state dumps written by oracle/ref_harness.cpp.

Each record holds, per body, the node kinematics and force components (Node.h:28-61), the rigid
body kinematics and forces (Body.h:46-95), works (Body.h:111-117), border lengths and contact
pressures, the neighbour list and the contact elements (Contact_Element.h:5-55)."""
from __future__ import annotations

import dataclasses
import struct
from typing import List

import numpy as np

MAGIC = 0x4D454C44
NODE_FIELDS = ["x", "u", "v", "a", "up", "vp", "ap", "f_int", "f_contact", "f_body", "f_dirichlet",
               "f_neumann", "f_damping", "f_total"]
CONTACT_INT = ["borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM",
               "nodeM0", "nodeM1", "nodeM2", "nodeM3", "shiftM0", "shiftM1", "shiftM2", "shiftM3", "nb_internal"]
CONTACT_DBL = ["shapeM0", "shapeM1", "shapeM2", "shapeM3", "gapn", "vgapn", "gapt", "vgapt", "xsi",
               "xnorm", "ynorm", "xtan", "ytan", "effective_mass", "length", "fx", "fy",
               "internal0", "internal1", "internal2"]
RIGID_FIELDS = ["cur", "disp", "vel", "acc", "f_contact", "f_body", "f_dirichlet", "f_neumann", "f_total"]


@dataclasses.dataclass
class BodyDump:
    rigid: bool
    nodes: dict            # field -> (n,2)
    rigid_state: dict      # field -> (3,)
    mass: float
    inertia: float
    works: np.ndarray      # (7,)
    border_length: List[np.ndarray]
    border_px: List[np.ndarray]
    border_py: List[np.ndarray]
    neighbours: np.ndarray # (k,3)
    contacts_i: np.ndarray # (c,16)
    contacts_d: np.ndarray # (c,20)


@dataclasses.dataclass
class Record:
    step: int
    tag: int
    time: float
    dt: float
    bodies: List[BodyDump]

    def contacts(self) -> dict:
        """All contact elements in list order with their slave body index added."""
        ci = [np.column_stack([np.full(b.contacts_i.shape[0], k, dtype=np.int32), b.contacts_i])
              for k, b in enumerate(self.bodies)]
        cd = [b.contacts_d for b in self.bodies]
        ci = np.concatenate(ci) if ci else np.zeros((0, 17), np.int32)
        cd = np.concatenate(cd) if cd else np.zeros((0, 20))
        out = {"bodyS": ci[:, 0]}
        for j, n in enumerate(CONTACT_INT):
            out[n] = ci[:, j + 1]
        for j, n in enumerate(CONTACT_DBL):
            out[n] = cd[:, j]
        return out

    def node_field(self, name: str) -> np.ndarray:
        return np.concatenate([b.nodes[name] for b in self.bodies])


def read_dump(path: str) -> List[Record]:
    data = open(path, "rb").read()
    off = 0
    out: List[Record] = []

    def ints(n):
        nonlocal off
        v = np.frombuffer(data, dtype=np.int32, count=n, offset=off)
        off += 4 * n
        return v

    def dbls(n):
        nonlocal off
        v = np.frombuffer(data, dtype=np.float64, count=n, offset=off)
        off += 8 * n
        return v

    while off < len(data):
        magic, step, tag = ints(3)
        assert magic == MAGIC, "corrupt dump"
        time, dt = dbls(2)
        nb = int(ints(1)[0])
        bodies = []
        for _ in range(nb):
            rigid, nn = (int(x) for x in ints(2))
            nd = dbls(28 * nn).reshape(nn, 14, 2)
            nodes = {f: nd[:, k, :].copy() for k, f in enumerate(NODE_FIELDS)}
            r = dbls(30)
            rs = {f: r[3 * k:3 * k + 3].copy() for k, f in enumerate(RIGID_FIELDS)}
            works = dbls(7).copy()
            nbd = int(ints(1)[0])
            bl, bpx, bpy = [], [], []
            for _ in range(nbd):
                nbn = int(ints(1)[0])
                bl.append(dbls(nbn).copy()); bpx.append(dbls(nbn).copy()); bpy.append(dbls(nbn).copy())
            nn_ = int(ints(1)[0])
            neigh = ints(3 * nn_).reshape(nn_, 3).copy()
            nc = int(ints(1)[0])
            ci = np.zeros((nc, 16), np.int32)
            cd = np.zeros((nc, 20))
            for k in range(nc):
                ci[k] = ints(16)
                cd[k] = dbls(20)
            bodies.append(BodyDump(bool(rigid), nodes, rs, float(r[27]), float(r[28]), works, bl, bpx, bpy,
                                   neigh, ci, cd))
        out.append(Record(int(step), int(tag), float(time), float(dt), bodies))
    return out
