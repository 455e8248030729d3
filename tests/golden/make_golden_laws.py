"""Generates tests/golden/laws_ref.json: the reference solver's own state for every case of
tests/test_oracle_laws.py (each contact law, with and without INITIALIZE_CZM where it applies,
NeoHookean, border conditions of deformable bodies, two 12-disc biaxial samples, an x-periodic
domain and a spinning rigid disc), at full FP64 precision.

    python tests/golden/make_golden_laws.py [case ...]
        (needs oracle/_ref/ref_harness, built by oracle/Makefile from the reference sources; with
        case names, only those cases are rerun and the others are kept from the existing file)

The harness (oracle/ref_harness.cpp) runs the reference's Load_static / Load_dynamic / set-up /
Euler_step / Update_proximity unchanged on one thread and dumps every node, work and contact
element; the fixture keeps SHA-256 digests per field and step, and the SHA-256 of each case's
generated input arrays."""
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

from conftest import input_checksum  # noqa: E402
from melody2d_b200 import generator as g  # noqa: E402
from oracle.refdump import read_dump  # noqa: E402
from test_oracle_laws import CASES, STEPS, case_scene, summary  # noqa: E402


def record_summary(r):
    node = {k: r.node_field(k) for k in ("x", "up", "f_int", "f_contact")}
    px = np.concatenate([p for b in r.bodies for p in b.border_px])
    py = np.concatenate([p for b in r.bodies for p in b.border_py])
    return summary(node, r.contacts(), np.array([b.works for b in r.bodies]), np.stack([px, py], axis=1))


def main():
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    out = os.path.join(HERE, "laws_ref.json")
    only = sys.argv[1:]
    cases = {}
    if only and os.path.exists(out):
        cases = json.load(open(out))["cases"]
    for name in CASES:
        if only and name not in only:
            continue
        sc = case_scene(name)
        flat = g.flatten(sc)
        with tempfile.TemporaryDirectory() as tmp:
            g.write_asc(sc, tmp)
            dump = os.path.join(tmp, "dump.bin")
            subprocess.run([harness, tmp, str(max(STEPS)), dump, "50", "1"], check=True, stdout=subprocess.DEVNULL)
            recs = read_dump(dump)
        by_step = {}
        for r in recs:
            if r.step in STEPS:
                by_step[r.step] = r      # the last record of a step is the post-proximity one
        cases[name] = {"input_sha256": input_checksum(flat),
                       "steps": {str(s): record_summary(by_step[s]) for s in STEPS}}
        print(name, "contacts", cases[name]["steps"][str(STEPS[-1])]["n_contacts"])
    cases = {k: cases[k] for k in CASES if k in cases}
    with open(out, "w") as fh:
        json.dump({"cases": cases}, fh, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
