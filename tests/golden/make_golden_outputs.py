"""Generates the reference-format output fixtures under tests/golden/outputs/: the files the reference
itself writes for the case conftest.outputs_scene() builds.

    python tests/golden/make_golden_outputs.py    (needs oracle/_ref/ref_harness, built by oracle/Makefile
                                                  from the reference sources)

1. oracle/ref_harness runs the reference's own loop on the case for 60 iterations with its output
   steps on (REF_OUTPUTS=1): Monitoring every iteration, Write_dynamic and Write_monitoring at the
   saves after iterations 30 and 60.  Kept: MONITORING.asc, DYNAMIC_00001.asc.gz, DYNAMIC_00002.asc.gz.
2. It then restarts from its own DYNAMIC_00001.asc (REF_RESTART=1) and runs 30 iterations; the final
   node kinematics, rigid bodies and works go to restart_ref.json at full FP64 precision (binary dump).
The SHA-256 of the generated input arrays is recorded so a change of the generator shows up as a
fixture mismatch rather than as a solver difference."""
import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import input_checksum, outputs_scene  # noqa: E402
from melody2d_b200 import generator as g  # noqa: E402
from oracle.refdump import read_dump  # noqa: E402

OUT = os.path.join(HERE, "outputs")
STEPS, RESTART_STEPS = 60, 30


def main():
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    scene = outputs_scene(STEPS)
    flat = g.flatten(scene)
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        case = os.path.join(tmp, "case")
        g.write_asc(scene, case)
        env = dict(os.environ, REF_OUTPUTS="1")
        subprocess.run([harness, case, str(STEPS), "-", "0", "1"], check=True, stdout=subprocess.DEVNULL, env=env)
        shutil.copy(os.path.join(case, "MONITORING.asc"), os.path.join(OUT, "MONITORING.asc"))
        for k in (1, 2):
            src = os.path.join(case, "DYNAMIC_%05d.asc" % k)
            with open(src, "rb") as fi, gzip.GzipFile(os.path.join(OUT, "DYNAMIC_%05d.asc.gz" % k), "wb", mtime=0) as fo:
                fo.write(fi.read())
        # restart from the reference's own file
        rcase = os.path.join(tmp, "restart")
        shutil.copytree(case, rcase)
        os.unlink(os.path.join(rcase, "MONITORING.asc"))
        dump = os.path.join(tmp, "restart.bin")
        env = dict(os.environ, REF_RESTART="1")
        subprocess.run([harness, rcase, str(RESTART_STEPS), dump, str(RESTART_STEPS), "1"], check=True,
                       stdout=subprocess.DEVNULL, env=env)
        recs = read_dump(dump)
    first, last = recs[0], [r for r in recs if r.step == RESTART_STEPS][-1]
    out = {"input_sha256": input_checksum(flat), "dt": float(flat["dt"]), "steps": STEPS,
           "restart_steps": RESTART_STEPS, "restart_time0": first.time, "restart_time": last.time}
    for name, r in (("restart_setup", first), ("restart_final", last)):
        out[name] = {f: np.concatenate([b.nodes[f] for b in r.bodies]).tolist() for f in ("x", "u", "v", "up", "vp")}
        out[name]["rigid"] = [np.concatenate([b.rigid_state[k] for k in ("cur", "disp", "vel")]).tolist()
                              for b in r.bodies if b.rigid]
        out[name]["works"] = [b.works.tolist() for b in r.bodies]
        out[name]["n_contacts"] = int(sum(len(b.contacts_i) for b in r.bodies))
    with open(os.path.join(OUT, "restart_ref.json"), "w") as fh:
        json.dump(out, fh)
    for f in sorted(os.listdir(OUT)):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
