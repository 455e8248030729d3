"""Pins the oracle to the reference solver.

tests/golden/lattice3x3_ref.json holds SHA-256 digests of the reference's own FP64 state (made by
tests/golden/make_golden.py with the reference compiled from its sources) after set-up and after
50 and 150 steps of a 3x3 squeezed lattice.  The oracle, run in its default mode (glibc pow, as the
reference), must reproduce every digest bit for bit.  Where the compiled reference is present
(oracle/_ref/ref_harness) a second, larger scene is compared directly."""
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, flat_of, input_checksum, squeezed_lattice

GOLDEN = os.path.join(ROOT, "tests", "golden", "lattice3x3_ref.json")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def oracle_summary(o, flat):
    st = o.node_state()
    f = o.forces()
    fields = {"x": o.positions(), "u": st[:, 0:2], "v": st[:, 2:4], "a": st[:, 4:6], "up": st[:, 6:8],
              "vp": st[:, 8:10], "ap": st[:, 10:12], "f_int": f["internal"], "f_contact": f["contact"]}
    out = {"node_" + k: sha(np.ascontiguousarray(v)) for k, v in fields.items()}
    rg, rf = o.rigid()
    rows = []
    for b in range(len(flat["body_type"])):
        if flat["body_type"][b] != 1:
            continue
        r = rg[b]
        rows.append(np.concatenate([r[7:10], r[10:13], r[13:16], r[16:19], rf[b][0:3], rf[b][6:9]]))
    out["rigid"] = sha(np.array(rows))
    out["rigid_values"] = np.array(rows)
    out["works"] = sha(o.works())
    c = o.contacts()
    cd = {k: c[k] for k in ("bodyS", "borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM",
                            "gapn", "gapt", "xsi", "xnorm", "ynorm", "fx", "fy")}
    cd["shapeM1"] = c["shapeM"][:, 1].copy()
    cd["shapeM2"] = c["shapeM"][:, 2].copy()
    for k, v in cd.items():
        out["contact_" + k] = sha(v.astype(np.float64))
    out["n_contacts"] = len(c)
    return out


def test_oracle_matches_reference_golden(oracle_built):
    from oracle.pyoracle import Oracle
    gold = json.load(open(GOLDEN))
    scene = squeezed_lattice(3, 3)
    flat = flat_of(scene)
    assert input_checksum(flat) == gold["input_sha256"], "generated input differs from the fixture's input"
    o = Oracle(flat, correctly_rounded=False)
    done = 0
    for step in sorted(int(s) for s in gold["steps"]):
        o.step(step - done)
        done = step
        ref = gold["steps"][str(step)]
        got = oracle_summary(o, flat)
        assert got["n_contacts"] == ref["n_contacts"], step
        np.testing.assert_array_equal(got["rigid_values"], np.array(ref["rigid_values"]), err_msg=f"rigid at {step}")
        for k, v in ref.items():
            if k in ("time", "n_contacts", "n_active", "rigid_values", "node_x_sample"):
                continue
            assert got[k] == v, f"{k} differs from the reference at step {step}"
        assert o.time == ref["time"]


def test_oracle_matches_compiled_reference_directly(oracle_built, tmp_path):
    """Runs the compiled reference (when present) on the 4x4 lattice and compares full arrays."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        pytest.skip("reference harness not built here (pinning relies on the committed golden digests)")
    from melody2d_b200 import generator as g
    from oracle.pyoracle import Oracle
    from oracle.refdump import read_dump
    scene = squeezed_lattice(4, 4)
    flat = flat_of(scene)
    g.write_asc(scene, str(tmp_path))
    dump = str(tmp_path / "d.bin")
    subprocess.run([harness, str(tmp_path), "60", dump, "30", "1"], check=True, stdout=subprocess.DEVNULL)
    recs = [r for r in read_dump(dump) if r.tag == 1 or r.step % 30 == 0]
    last = {}
    for r in recs:
        last[r.step] = r
    o = Oracle(flat)
    done = 0
    for step in (0, 30, 60):
        o.step(step - done)
        done = step
        r = last[step]
        np.testing.assert_array_equal(o.positions(), r.node_field("x"))
        np.testing.assert_array_equal(o.node_state()[:, 6:8], r.node_field("up"))
        np.testing.assert_array_equal(o.forces()["contact"], r.node_field("f_contact"))
        c = o.contacts(); rc = r.contacts()
        np.testing.assert_array_equal(c["fx"], rc["fx"])
        np.testing.assert_array_equal(c["segmentM"], rc["segmentM"])
