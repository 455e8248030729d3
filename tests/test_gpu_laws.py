"""Every contact law, the NeoHookean material and the border conditions of deformable bodies
against the oracle.

The contact laws (Code/Model.h:81-506) use only +, -, *, / and sqrt, which round the same way on
the GPU and on the host, so with each law the FP64 trajectory of a 3x3 lattice pressed by its
plates (about 45 loaded contacts, grain-grain and grain-plate, after 100 steps) is bit-identical
to the oracle's correctly-rounded mode: node kinematics, contact list with history and internal
variables, rigid state, works.

Soft Dirichlet, oriented and following Neumann conditions on deformable borders (the plates and
walls of the other tests carry driven and oriented conditions on rigid bodies) are bit-identical
as well: force components after one step and the trajectory over 100 steps.

The NeoHookean update (Code/Model.h:52-73) evaluates J^(-5/3) with pow, whose last bit differs
between CUDA's and glibc's implementations.  Stated tolerances: FP64 node state within 1e-9 of the
largest displacement after 100 steps and the same active contacts; the mixed-precision form's
kinetic energy and wall forces within 1e-5 relative after 200 steps."""
import numpy as np
import pytest

from test_gpu_parity import assert_contacts_equal

pytestmark = pytest.mark.gpu

# file parameters per law type (MEL_LAW_*, Code/IO.h:775-783), sized against the lattice's contact
# loads (kn * overlap ~ 1e4) so that the strength limits are reached
LAWS = {
    0: [1e10],                                                    # Frictionless: kn
    1: [1e10, 1e9, 2e3, 2e3],                                     # Cohesion: kn, kt, gtang, gtens
    2: [1e10, 1e9, 0.3, 0.0, 0.0],                                # MohrCoulomb: kn, kt, fric, coh, tens
    3: [1e10, 1e9, 0.3, 0.0, 0.0, 0.2],                           # DampedMohrCoulomb: ..., damping
    4: [1e10, 1e9, 0.3, 0.0, 0.0, 0.5],                           # TwoSlopesMohrCoulomb: ..., unloading ratio
    5: [1e10, 1e9, 2e10, 0.5, 4e3, 4e3, 0.3, 0.0, 0.0, 0.05],     # BondedMohrCoulomb
    6: [1e10, 4e3, 1e-6, 1e3, 1.0],                               # CzmLinear: kini, Pnlim, gapnlim, Pnres, NTratio
    7: [1e10, 4e3, 1e-6, 1e3, 1.0, 2e3, 0.01, 0.01],              # CzmFatigue: ..., Pnfat, Raten, Ratet
}


def flat_with(law_type=None, params=None, neohookean=False):
    from melody2d_b200 import generator as g
    sc = g.disc_lattice_scene(seed=0, nx=3, ny=3, pitch=2.0e-3, gap0=-1e-6, nsteps=300, v_plate=0.05)
    if law_type is not None:
        sc.laws = [(m1, m2, law_type, 0, list(params)) for (m1, m2, _, _, _) in sc.laws]
    if neohookean:
        sc.materials = [(name, 1 if name == "Grain" else t, p) for (name, t, p) in sc.materials]
    return g.flatten(sc)


@pytest.mark.parametrize("law", sorted(LAWS))
def test_contact_law_bit_identical(gpu_lib, oracle_built, law):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_with(law, LAWS[law])
    assert set(np.asarray(flat["law_type"]).tolist()) == {law}
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    for _ in range(5):
        g.step(20)
        o.step(20)
        np.testing.assert_array_equal(g.node_state(), o.node_state())
        assert_contacts_equal(g.contacts(), o.contacts())
    np.testing.assert_array_equal(g.rigid()[0], o.rigid()[0])
    np.testing.assert_array_equal(g.works(), o.works())
    assert (g.contacts()["fx"] != 0).sum() > 20
    g.close()


def test_neohookean_fp64_within_tolerance(gpu_lib, oracle_built):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_with(neohookean=True)
    assert 1 in np.asarray(flat["material_type"]).tolist()
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    g.step(100)
    o.step(100)
    sg, so = g.node_state(), o.node_state()
    scale = np.abs(so[:, 6:8]).max()
    assert scale > 0
    assert np.abs(sg[:, 6:8] - so[:, 6:8]).max() <= 1e-9 * scale
    assert g.monitor().active_contacts == o.monitor().active_contacts
    g.close()


def test_neohookean_mixed_within_tolerance(gpu_lib, oracle_built):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_with(neohookean=True)
    g = Solver.from_flat(flat, precision=1)
    o = Oracle(flat, correctly_rounded=True)
    g.step(200)
    o.step(200)
    mg, mo = g.monitor(), o.monitor()

    def rel(a, b):
        a, b = np.asarray(a, float), np.asarray(b, float)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    assert rel(mg.kinetic_energy, mo.kinetic_energy) <= 1e-5
    assert rel(list(mg.rigid_force), list(mo.rigid_force)) <= 1e-5
    assert mg.active_contacts == mo.active_contacts
    g.close()


def flat_with_border_conditions():
    """The pressed 3x3 lattice with border conditions on three of its deformable discs: soft
    Dirichlet, oriented Neumann and following Neumann in both directions (Body::Update_bc_forces,
    Code/Body.h:669-799)."""
    from melody2d_b200 import generator as g
    sc = g.disc_lattice_scene(seed=0, nx=3, ny=3, pitch=2.0e-3, gap0=-1e-6, nsteps=300, v_plate=0.05)
    hist = lambda v: (np.array([0.0, g.T_HIST_END]), np.array([v, v]))
    combos = [((g.BC_SOFT, (1e8, 1e2), hist(0.02)), (g.BC_ORIENTED, (0.0, 0.0), hist(-2e4))),
              ((g.BC_FOLLOWING, (0.0, 0.0), hist(3e4)), (g.BC_SOFT, (5e7, 0.0), hist(-0.01))),
              ((g.BC_ORIENTED, (0.0, 0.0), hist(1e4)), (g.BC_FOLLOWING, (0.0, 0.0), hist(-1e4)))]
    for body, bc in zip(sc.bodies[:3], combos):
        assert body.kind == "deformable"
        body.borders[0]["bc"] = list(bc)
    return g.flatten(sc)


def test_deformable_border_conditions_bit_identical(gpu_lib, oracle_built):
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    flat = flat_with_border_conditions()
    g = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    g.record_forces(True)
    g.step(1)
    o.step(1)
    fg, fo = g.forces(), o.forces()
    for k in ("neumann", "dirichlet", "internal", "contact", "total"):
        np.testing.assert_array_equal(fg[k], fo[k], err_msg=k)
    assert np.abs(fo["neumann"]).max() > 0 and np.abs(fo["dirichlet"]).max() > 0
    for _ in range(5):
        g.step(20)
        o.step(20)
        np.testing.assert_array_equal(g.node_state(), o.node_state())
        assert_contacts_equal(g.contacts(), o.contacts())
    np.testing.assert_array_equal(g.works(), o.works())
    g.close()


@pytest.mark.parametrize("case", ["law5+czm", "law6+czm", "law7+czm"])
def test_initialize_czm_bit_identical(gpu_lib, oracle_built, case):
    """INITIALIZE_CZM (Code/Proximity.h:481-541) bonds the set-up contacts closer than the law's
    initial-gap parameter; the bonded and damage branches of BondedMohrCoulomb, CZMlinear and
    CZMfatigue then run bit-identically to the oracle (itself pinned to the compiled reference on
    these cases, tests/test_oracle_laws.py)."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    flat = g.flatten(case_scene(case))
    assert int(np.asarray(flat["flags"])[3]) == 1
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    assert_contacts_equal(gs.contacts(), o.contacts())
    assert (o.contacts()["internal"][:, 0] == 0).sum() > 10, "the scenario must start with bonded contacts"
    for _ in range(5):
        gs.step(20)
        o.step(20)
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    np.testing.assert_array_equal(gs.works(), o.works())
    gs.close()


def test_damping_matrices_bit_identical(gpu_lib, oracle_built):
    """Rayleigh damping matrices on the grains (MATRICES of STATIC_DATA, applied by
    Body::Update_damping_forces, Code/Body.h:1057-1154, to the velocity parameters): node state,
    contacts and works equal the oracle's (itself pinned to the compiled reference on this case,
    tests/test_oracle_laws.py) over 100 steps, and the damping work is non-zero."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    flat = g.flatten(case_scene("damping"))
    assert len(flat["matrix_damping"]) > 1000
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    for _ in range(5):
        gs.step(20)
        o.step(20)
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    np.testing.assert_array_equal(gs.works(), o.works())
    assert np.abs(gs.works()[:, 5]).max() > 0
    gs.close()


def test_alid_layers_bit_identical(gpu_lib, oracle_built):
    """ALID absorbing layers on the grains (the ALID block of STATIC_CONTROL with x and y histories
    of the layer's reference velocity, Body::Update_alid_forces, Code/Body.h:1163-1296): node state,
    contacts and works equal the oracle's (itself pinned to the compiled reference on this case,
    tests/test_oracle_laws.py) over 100 steps; the ALID work is non-zero, and the model with its
    layers read from the case's files by the library's loader steps to the same state."""
    import tempfile
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    scene = case_scene("alid")
    flat = g.flatten(scene)
    assert np.count_nonzero(flat["node_alid"]) > 100
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    for _ in range(5):
        gs.step(20)
        o.step(20)
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    np.testing.assert_array_equal(gs.works(), o.works())
    assert np.abs(gs.works()[:, 6]).max() > 0
    with tempfile.TemporaryDirectory() as tmp:
        g.write_asc(scene, tmp)
        gf = Solver.from_files(tmp)
        gf.step(100)
        np.testing.assert_array_equal(gf.node_state(), gs.node_state())
        gf.close()
    gs.close()


def test_material_matrix_updates_bit_identical(gpu_lib, oracle_built):
    """UPDATE_MASS_MATRIX, UPDATE_STIFFNESS_MATRIX and UPDATE_DAMPING_MATRIX (Body::Update_material,
    Code/Body.h:2708-2875) on grains with ALID layers: the file's matrices come from half the
    grains' modulus and carry no damping, and the set-up rebuilds masses, stiffness (which the ALID
    coupling terms use) and Rayleigh damping from the material.  Node state, contacts and works
    equal the oracle's (itself pinned to the compiled reference on this case) over 100 steps, the
    damping work is non-zero, and the model read from the case's files steps to the same state."""
    import tempfile
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    scene = case_scene("update_matrices")
    flat = g.flatten(scene)
    assert list(flat["flags"][4:7]) == [1, 1, 1] and np.abs(flat["matrix_damping"]).max() == 0
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    for _ in range(5):
        gs.step(20)
        o.step(20)
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    np.testing.assert_array_equal(gs.works(), o.works())
    assert np.abs(gs.works()[:, 5]).max() > 0 and np.abs(gs.works()[:, 6]).max() > 0
    with tempfile.TemporaryDirectory() as tmp:
        g.write_asc(scene, tmp)
        gf = Solver.from_files(tmp)
        gf.step(100)
        np.testing.assert_array_equal(gf.node_state(), gs.node_state())
        gf.close()
    gs.close()


def test_damage_deactivation_and_monitoring(gpu_lib, oracle_built):
    """Damage (Body::Update_damage, Code/Body.h:2667-2700) on bonded contacts.  DEACTIVATION on
    damage: the free rigid disc (no contact, damage 1) turns inactive at the first update and the
    loaded discs' entries never hold, as in the oracle (pinned to the compiled reference on this
    case); the trajectories stay bit-identical.  Monitoring's Damage entries (Monitoring.h:385-390)
    of two loaded discs, one row per step, equal the oracle's Update_damage evaluated where
    Monitoring runs (after each step, before its proximity update), bit for bit, and vary."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    flat = g.flatten(case_scene("deactivation_damage"))
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    gs.monitor_setup([[8, 0], [8, 4]], ring_rows=200, first_iteration=0)
    o.monitor_damage([0, 4], cap=200)
    for _ in range(10):
        gs.step(10)
        o.step(10)
        np.testing.assert_array_equal(gs.body_status(), o.body_status())
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
    rows = gs.monitor_rows()
    got = np.array([r[6:8] for r in rows])
    want = o.damage_log()
    assert got.shape == want.shape == (100, 2)
    np.testing.assert_array_equal(got, want)
    assert len(np.unique(got[:, 1])) > 1 and got.min() < 1.0
    assert np.nonzero(gs.body_status() == 1)[0].tolist() == [11]
    gs.close()


def test_deactivation_bit_identical(gpu_lib, oracle_built):
    """DEACTIVATION entries (Update_status after each proximity update, Code/Proximity.h:550-1007):
    a free rigid disc beside the pressed lattice turns inactive by its displacement at the same
    proximity update as in the oracle (pinned to the compiled reference on this case,
    tests/test_oracle_laws.py) and stops; the entries that never hold (speed, node position, summed
    total force of a loaded disc) are evaluated at every update; the trajectories stay
    bit-identical."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    from oracle.pyoracle import Oracle
    from test_oracle_laws import case_scene
    flat = g.flatten(case_scene("deactivation"))
    gs = Solver.from_flat(flat)
    o = Oracle(flat, correctly_rounded=True)
    seen = set()
    for _ in range(10):
        gs.step(10)
        o.step(10)
        np.testing.assert_array_equal(gs.body_status(), o.body_status())
        np.testing.assert_array_equal(gs.node_state(), o.node_state())
        assert_contacts_equal(gs.contacts(), o.contacts())
        seen |= set(np.nonzero(gs.body_status() == 1)[0].tolist())
    np.testing.assert_array_equal(gs.works(), o.works())
    assert seen == {11}, seen
    gs.close()
