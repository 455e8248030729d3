"""Reference-format output boundary, host side (no GPU): the MONITORING list parser
(Read_spy_line, Code/IO.h:11-590) and the run counters read by mel_load_run_control, and the
library's loader reading a DYNAMIC file the reference itself wrote (Write_dynamic, Code/IO.h:2351)
when a run restarts from it (argv[1] of Code/main.cpp).  Fixtures: tests/golden/outputs/, written
by tests/golden/make_golden_outputs.py from the reference's own run."""
import gzip
import json
import os
import shutil

import numpy as np
import pytest

from conftest import input_checksum, outputs_scene

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "outputs")

# the vectors Read_spy_line builds for conftest.outputs_scene()'s MONITORING lines
EXPECTED = {
    "Position Y 4 -1": [0, 1, 4, -1], "Position X 0 -1": [0, 0, 0, -1], "Position Y 1 7": [0, 1, 1, 7],
    "Displacement Mag 1 5": [1, 2, 1, 5], "Displacement R 5 -1": [1, 3, 5, -1], "Velocity Y 5 -1": [2, 1, 5, -1],
    "Velocity X 3 -1": [2, 0, 3, -1], "Acceleration X 2 -1": [3, 0, 2, -1], "Acceleration Mag 4 -1": [3, 2, 4, -1],
    "Force Y Contact 4 -1": [4, 1, 2, 4, -1], "Force X Total 0 3": [4, 0, 0, 0, 3],
    "Force Mag Internal 1 2": [4, 2, 1, 1, 2], "Force X Body 2 4": [4, 0, 3, 2, 4],
    "Force Y Dirichlet 5 -1": [4, 1, 4, 5, -1], "Force Y Neumann 0 1": [4, 1, 5, 0, 1],
    "Contact Gapn 0 0 7": [7, 0, 0, 0, 7], "Contact Xnorm 1 0 3": [7, 3, 1, 0, 3], "Energy Kinetic 0": [9, 0, 0],
    "Energy Kinetic 4": [9, 0, 4], "Energy Kinetic -1": [9, 0, -1], "Energy Deformation 1": [9, 1, 1],
    "Work Contact 0": [10, 1, 0], "Work Dirichlet -1": [10, 3, -1], "Work Internal 5": [10, 0, 5],
    "Error X 0 1": [11, 0, 0, 1], "Position AllX": [0, 6],
}


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    from melody2d_b200 import generator as g
    sc = outputs_scene(60)
    d = str(tmp_path_factory.mktemp("outputs_case"))
    g.write_asc(sc, d)
    with gzip.open(os.path.join(GOLD, "DYNAMIC_00001.asc.gz"), "rb") as fi, \
            open(os.path.join(d, "DYNAMIC_00001.asc"), "wb") as fo:
        shutil.copyfileobj(fi, fo)
    return sc, d


def test_fixture_inputs_match_generator():
    from melody2d_b200 import generator as g
    ref = json.load(open(os.path.join(GOLD, "restart_ref.json")))
    assert input_checksum(g.flatten(outputs_scene(60))) == ref["input_sha256"]


def test_monitoring_list_and_counters(case):
    from melody2d_b200.solver import load_run_control
    sc, d = case
    rc = load_run_control(d, 0)
    assert rc["simulation_name"] == "outputs"
    assert rc["number_save"] == 0 and rc["number_iteration"] == 0
    assert rc["save_period"] == sc.save_period and rc["print_period"] == sc.print_period
    assert rc["next_save"] == sc.save_period and rc["next_print"] == sc.print_period
    assert rc["flags"][1] == 1 and rc["flags"][8] == 0            # MONITOR_ENERGY, monitoring on
    big = [ln for ln in sc.monitored if ln.startswith("Force X Contact")][0]
    expected = dict(EXPECTED, **{big: [4, 0, 2, int(big.split()[3]), -1]})
    mon = rc["monitored"]
    assert mon.shape == (len(sc.monitored), 7)
    for line, row in zip(sc.monitored, mon):
        want = np.zeros(7)
        want[:len(expected[line])] = expected[line]
        np.testing.assert_array_equal(row, want, err_msg=line)


def test_loader_reads_reference_dynamic(case):
    """Restart input: the state the reference wrote after 30 iterations, as the library's loader
    reads it, equals the state the reference itself reads back from the same file (its restart's
    set-up record, which leaves these fields untouched)."""
    from melody2d_b200.solver import load_desc_arrays, load_run_control
    _, d = case
    ref = json.load(open(os.path.join(GOLD, "restart_ref.json")))
    flat = load_desc_arrays(d, 1)
    st = flat["node_state"].reshape(-1, 12)
    setup = ref["restart_setup"]
    for k, col in (("u", 0), ("v", 2), ("up", 6), ("vp", 8)):
        np.testing.assert_array_equal(st[:, col:col + 2], np.array(setup[k]), err_msg=k)
    assert flat["time"] == ref["restart_time0"]
    rc = load_run_control(d, 1)
    assert rc["number_save"] == 1 and rc["number_iteration"] == 30
    assert rc["number_print"] == 1
