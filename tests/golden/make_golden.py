"""Generates tests/golden/lattice3x3_ref.json: the reference solver's own state, run on a generated
3x3 lattice, at full FP64 precision.

    python tests/golden/make_golden.py        (needs oracle/_ref/ref_harness, built by oracle/Makefile
                                              from the reference sources)

The harness (oracle/ref_harness.cpp) runs the reference's Load_static / Load_dynamic / set-up /
Euler_step / Update_proximity unchanged on one thread and dumps every node, rigid body, work and
contact element.  The fixture keeps a SHA-256 per field and step (bit-exact comparison) plus a few
summary numbers for diagnostics, and the SHA-256 of the generated input arrays."""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import input_checksum, squeezed_lattice, flat_of  # noqa: E402
from melody2d_b200 import generator as g  # noqa: E402
from oracle.refdump import read_dump  # noqa: E402

STEPS = [0, 50, 150]
NODE_FIELDS = ["x", "u", "v", "a", "up", "vp", "ap", "f_int", "f_contact"]
CONTACT_KEYS = ["bodyS", "borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM",
                "gapn", "gapt", "xsi", "xnorm", "ynorm", "fx", "fy", "shapeM1", "shapeM2"]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def record_summary(r):
    out = {"time": r.time}
    for f in NODE_FIELDS:
        a = r.node_field(f)
        out["node_" + f] = sha(a)
    out["node_x_sample"] = r.node_field("x")[::97].tolist()
    rig = np.array([np.concatenate([b.rigid_state[k] for k in ("cur", "disp", "vel", "acc", "f_contact", "f_dirichlet")])
                    for b in r.bodies if b.rigid])
    out["rigid"] = sha(rig)
    out["rigid_values"] = rig.tolist()
    out["works"] = sha(np.array([b.works for b in r.bodies]))
    c = r.contacts()
    out["n_contacts"] = int(len(c["fx"]))
    out["n_active"] = int(np.sum((c["fx"] != 0) | (c["fy"] != 0)))
    for k in CONTACT_KEYS:
        out["contact_" + k] = sha(c[k].astype(np.float64) if c[k].dtype != np.float64 else c[k])
    return out


def main():
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    scene = squeezed_lattice(3, 3)
    flat = flat_of(scene)
    with tempfile.TemporaryDirectory() as tmp:
        g.write_asc(scene, tmp)
        dump = os.path.join(tmp, "dump.bin")
        subprocess.run([harness, tmp, str(max(STEPS)), dump, "50", "1"], check=True, stdout=subprocess.DEVNULL)
        recs = read_dump(dump)
    by_step = {}
    for r in recs:
        if r.step in STEPS:
            by_step[r.step] = r          # the last record of a step is the post-proximity one
    fixture = {"input_sha256": input_checksum(flat), "dt": float(flat["dt"]),
               "steps": {str(s): record_summary(by_step[s]) for s in STEPS}}
    with open(os.path.join(HERE, "lattice3x3_ref.json"), "w") as fh:
        json.dump(fixture, fh, indent=1)
    print("wrote", os.path.join(HERE, "lattice3x3_ref.json"))


if __name__ == "__main__":
    main()
