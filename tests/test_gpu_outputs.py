"""Reference-format outputs from the GPU: the melody_gpu host loop writes MONITORING.asc and
DYNAMIC_nnnnn.asc (Monitoring, Code/Monitoring.h:8-559; Write_monitoring and Write_dynamic,
Code/IO.h:2351-2668) that match the files the reference itself wrote for the same case; a run
restarts from a DYNAMIC file the reference wrote and follows the reference's own restart; and the
device monitoring's per-body quantities equal the reference's arithmetic on the same state bit for
bit.  Fixtures: tests/golden/outputs/ (tests/golden/make_golden_outputs.py)."""
import gzip
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import outputs_scene

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "outputs")
EXE = os.path.join(os.path.dirname(HERE), "melody2d_b200", "melody_gpu")
# the files keep 10 significant digits; the GPU follows the correctly rounded x^-1/2 where the
# reference calls glibc's pow (a few units in the last place per call), so a printed value may
# differ by one unit in its 10th digit, and values that cancel (accelerations, force sums) by a
# small fraction of their column's scale
REL, ABS_OF_SCALE = 2e-9, 1e-10


def _case(tmp_path, with_restart=False):
    from melody2d_b200 import generator as g
    sc = outputs_scene(60)
    d = str(tmp_path / "case")
    g.write_asc(sc, d)
    if with_restart:
        with gzip.open(os.path.join(GOLD, "DYNAMIC_00001.asc.gz"), "rb") as fi, \
                open(os.path.join(d, "DYNAMIC_00001.asc"), "wb") as fo:
            shutil.copyfileobj(fi, fo)
    return sc, d


def _num(tok):
    try:
        return float(tok)
    except ValueError:
        return None


def _compare_tables(got_lines, ref_lines, what):
    """Token-by-token comparison; numeric tokens within REL of the value plus ABS_OF_SCALE of the
    largest magnitude in the same column of the same kind of line."""
    assert len(got_lines) == len(ref_lines), (what, len(got_lines), len(ref_lines))
    got = [ln.split() for ln in got_lines]
    ref = [ln.split() for ln in ref_lines]
    scale = {}
    for r in ref:
        for j, t in enumerate(r):
            v = _num(t)
            if v is not None:
                k = (len(r), j)
                scale[k] = max(scale.get(k, 0.0), abs(v))
    worst = 0.0
    for i, (a, b) in enumerate(zip(got, ref)):
        assert len(a) == len(b), (what, i, a, b)
        for j, (x, y) in enumerate(zip(a, b)):
            vy = _num(y)
            if vy is None:
                assert x == y, (what, i, j, x, y)
                continue
            vx = _num(x)
            assert vx is not None, (what, i, j, x, y)
            tol = REL * abs(vy) + ABS_OF_SCALE * scale[(len(b), j)]
            assert abs(vx - vy) <= tol, (what, "line", i, "token", j, x, y)
            if tol > 0:
                worst = max(worst, abs(vx - vy) / tol)
    return worst


def test_melody_gpu_writes_the_reference_files(tmp_path, gpu_lib):
    _, d = _case(tmp_path)
    r = subprocess.run([EXE, "0", d, "1000"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    with open(os.path.join(d, "MONITORING.asc")) as fh:
        got = fh.read().splitlines()
    with open(os.path.join(GOLD, "MONITORING.asc")) as fh:
        ref = fh.read().splitlines()
    assert len(ref) == 60
    w = _compare_tables(got, ref, "MONITORING.asc")
    print("MONITORING.asc worst |diff|/tol", w)
    for k in (1, 2):
        with open(os.path.join(d, "DYNAMIC_%05d.asc" % k)) as fh:
            got = fh.read().splitlines()
        with gzip.open(os.path.join(GOLD, "DYNAMIC_%05d.asc.gz" % k), "rt") as fh:
            ref = fh.read().splitlines()
        w = _compare_tables(got, ref, "DYNAMIC_%05d.asc" % k)
        print("DYNAMIC_%05d.asc worst |diff|/tol" % k, w)


def test_restart_from_a_reference_dynamic_file(tmp_path, gpu_lib):
    from melody2d_b200.solver import Solver
    _, d = _case(tmp_path, with_restart=True)
    ref = json.load(open(os.path.join(GOLD, "restart_ref.json")))
    s = Solver.from_files(d, restart_index=1)
    try:
        t0, _ = s.time()
        assert t0 == ref["restart_time0"]
        s.step(ref["restart_steps"])
        t1, _ = s.time()
        assert t1 == ref["restart_time"]
        st = s.node_state()
        fin = ref["restart_final"]
        for k, col in (("u", 0), ("v", 2), ("up", 6), ("vp", 8)):
            want = np.array(fin[k])
            got = st[:, col:col + 2]
            tol = 1e-9 * np.abs(want).max()
            assert np.abs(got - want).max() <= tol, (k, np.abs(got - want).max(), tol)
        rg = s.rigid()[0]
        rig = np.array(fin["rigid"])
        from melody2d_b200 import abi
        got = np.array([np.concatenate([rg[b, abi_idx:abi_idx + 3] for abi_idx in (7, 10, 13)])
                        for b in range(rg.shape[0]) if b >= 4])
        assert np.abs(got - rig).max() <= 1e-9 * max(np.abs(rig).max(), 1e-30)
        assert s.contacts().shape[0] == fin["n_contacts"]
    finally:
        s.close()


def test_device_monitoring_equals_reference_arithmetic(tmp_path, gpu_lib):
    """Entries of one node or one body: the row's value equals the reference's expression
    (Code/Monitoring.h) evaluated on the same state in the same order, bit for bit."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    sc = outputs_scene(60)
    flat = g.flatten(sc)
    s = Solver.from_flat(flat)
    try:
        entries = [[0, 1, 4, -1], [0, 0, 0, -1], [0, 1, 1, 7], [1, 2, 1, 5], [2, 1, 3, -1], [3, 0, 2, -1],
                   [9, 0, 0], [9, 0, 4], [10, 1, 0], [10, 3, -1], [7, 0, 0, 0, 7]]
        s.monitor_setup(entries, ring_rows=64, first_iteration=0)
        s.step(25)
        rows = s.monitor_rows()
        assert len(rows) == 25
        row = rows[-1]
        st = s.node_state()
        x = s.positions()
        rg = s.rigid()[0]
        w = s.works()
        m = flat["node_mass"].reshape(-1, 2)
        ptr = flat["body_node_ptr"]
        t, dt = s.time()
        assert row[0] == 25 and row[1] == t and row[2] == dt and list(row[3:6]) == [0, 0, 0]

        def mean(a, b):
            sx = sy = sm = 0.0
            for j in range(ptr[b], ptr[b + 1]):
                sx += a[j, 0] * m[j, 0]
                sy += a[j, 1] * m[j, 1]
                sm += m[j, 0]
            return sx / sm, sy / sm

        want = [rg[4, 8], mean(x, 0)[0], x[ptr[1] + 7, 1]]
        u = st[ptr[1] + 5, 0:2]
        want.append((u[0] * u[0] + u[1] * u[1]) ** 0.5)
        want.append(mean(st[:, 2:4], 3)[1])
        want.append(mean(st[:, 4:6], 2)[0])
        ke = 0.0
        for j in range(ptr[0], ptr[1]):
            ke += 0.5 * st[j, 8] * st[j, 8] * m[j, 0]
            ke += 0.5 * st[j, 9] * st[j, 9] * m[j, 1]
        want.append(ke)
        kr = 0.0
        kr += 0.5 * rg[4, 13] * rg[4, 13] * rg[4, 3]
        kr += 0.5 * rg[4, 14] * rg[4, 14] * rg[4, 3]
        kr += 0.5 * rg[4, 15] * rg[4, 15] * rg[4, 4]
        want.append(kr)
        want.append(w[0, 1])
        sw = 0.0
        for b in range(w.shape[0]):
            sw += w[b, 3]
        want.append(sw)
        c = s.contacts()
        hit = [k for k in range(len(c)) if c["bodyS"][k] == 0 and c["borderS"][k] == 0 and c["border_nodeS"][k] == 7]
        if hit:
            want.append(c["gapn"][hit[0]])
        assert len(row) == 6 + len(want)
        np.testing.assert_array_equal(row[6:], np.array(want))
    finally:
        s.close()
