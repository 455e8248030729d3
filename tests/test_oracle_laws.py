"""Pins the oracle to the reference solver for every contact law, the NeoHookean material, the
border conditions of deformable bodies, INITIALIZE_CZM, two 12-disc biaxial samples (rigid
plates driven, lateral walls under oriented pressure along long borders, rigid-rigid pairs), an
x-periodic domain (discs meeting across the seam, "Periodic" rigid strips) and a free rigid disc
spinning among deformable discs (rigid rotation through cos and sin).

tests/golden/laws_ref.json holds SHA-256 digests of the reference's own FP64 state (made by
tests/golden/make_golden_laws.py with the reference compiled from its sources) after set-up and
after 50 and 100 steps of each case (a 3x3 lattice pressed by its plates, or a biaxial sample).  The oracle, run in
its default mode (glibc pow, as the reference), must reproduce every digest bit for bit: node
positions, displacement parameters, internal and contact forces, and every contact element with
its history and internal variables.  The GPU is pinned to the oracle on the same cases by
tests/test_gpu_laws.py.

Law parameters are complete as the reference's loader reads them (Code/IO.h:700-790); the last
parameter of BondedMohrCoulomb, CZMlinear and CZMfatigue is the initial-gap threshold that
INITIALIZE_CZM uses to bond the set-up contacts (Code/Proximity.h:481-545)."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, input_checksum

GOLDEN = os.path.join(ROOT, "tests", "golden", "laws_ref.json")
STEPS = [0, 50, 100]

# file parameters per law type (MEL_LAW_*), complete as Load_static reads them
LAW_PARAMS = {
    0: [1e10],
    1: [1e10, 1e9, 2e3, 2e3],
    2: [1e10, 1e9, 0.3, 0.0, 0.0],
    3: [1e10, 1e9, 0.3, 0.0, 0.0, 0.2],
    4: [1e10, 1e9, 0.3, 0.0, 0.0, 0.5],
    5: [1e10, 1e9, 2e10, 0.5, 4e3, 4e3, 0.3, 0.0, 0.0, 0.05, 1e-6],
    6: [1e10, 4e3, 1e-6, 1e3, 1.0, 1e-6],
    7: [1e10, 4e3, 1e-6, 1e3, 1.0, 2e3, 0.01, 0.01, 1e-6],
}

CASES = [f"law{l}" for l in sorted(LAW_PARAMS)] + ["law5+czm", "law6+czm", "law7+czm", "neohookean",
                                                    "border_conditions", "biaxial12_s5", "biaxial12_s7",
                                                    "periodic", "rotor", "adaptive_euler", "euler_2",
                                                    "mass_scaling", "adaptive_mass_scaling", "damping",
                                                    "deactivation", "alid", "deactivation_damage",
                                                    "update_matrices"]

# Solver_step schemes (Code/Solver.h:98-486) with their parameters: Target_error, Control_parameter,
# Accepted_ratio, Max_mass_scaling, Control_parameter_mass_scaling, Error_factor_mass_scaling,
# Decrease_factor_mass_scaling (Code/IO.h:821-893)
SOLVER_CASES = {"adaptive_euler": (1, (2e-3, 0.2, 0.9)), "euler_2": (4, (2e-3, 0.2, 0.9)),
                "mass_scaling": (2, (2e-3, 0.2, 0.9, 50.0, 1.0, 0.5, 0.99)),
                "adaptive_mass_scaling": (3, (2e-3, 0.2, 1.0, 50.0, 1.0, 0.5, 0.99))}


def case_scene(name):
    """The scene of one case: a biaxial sample, or the pressed 3x3 lattice (about 45 loaded
    contacts after 100 steps) with the case's law, material or border conditions."""
    from melody2d_b200 import generator as g
    if name == "periodic":
        return g.periodic_strip_scene()
    if name == "rotor":
        return g.rotor_scene()
    if name.startswith("biaxial12_s"):
        return g.biaxial_scene(seed=int(name.split("_s")[1]), n_discs=12, n_border=32, n_interior=80, workers=1)
    sc = g.disc_lattice_scene(seed=0, nx=3, ny=3, pitch=2.0e-3, gap0=-1e-6, nsteps=300, v_plate=0.05)
    if name.startswith("law"):
        law = int(name[3])
        sc.laws = [(m1, m2, law, 0, list(LAW_PARAMS[law])) for (m1, m2, _, _, _) in sc.laws]
        sc.initialize_czm = name.endswith("+czm")
    elif name in SOLVER_CASES:
        solver, prm = SOLVER_CASES[name]
        sc.solver = solver
        sp = list(sc.solver_params)
        sp[:len(prm)] = prm
        sc.solver_params = tuple(sp)
    elif name == "deactivation":
        # Update_status after each proximity update: a free rigid disc flying beside the pressed
        # lattice (body 11) turns inactive by its displacement at step 50 and stops; the other
        # entries (speed, node position, summed total force of a loaded disc) are evaluated at
        # every update and never hold
        xmax = max(b.nodes[:, 0].max() for b in sc.bodies)
        ymid = 0.5 * (min(b.nodes[:, 1].min() for b in sc.bodies) + max(b.nodes[:, 1].max() for b in sc.bodies))
        h = 2.0 * np.pi * 0.8e-3 / 32
        sc.bodies.append(g.make_rigid_disc((xmax + 4e-3, ymid), 0.8e-3, 32, 1, 7800.0, 0.5 * h, 0.5 * h,
                                           velocity=(0.01, 0.0)))
        sc.deactivation = ["Displacement X 11 -1 above 2e-7", "Velocity Mag 4 -1 above 100",
                           "Position Y 3 5 below -1", "Force Y Total 0 -1 above 1e9",
                           "Velocity X 8 -1 equal 12345"]
    elif name == "damping":
        # Rayleigh damping matrices on the grains (MATRICES, Body::Update_damping_forces)
        E, nu = 1e8, 0.3
        g.add_damping(sc, 0.02 * sc.dt, 0.05 / sc.dt, E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu)))
    elif name == "deactivation_damage":
        # Update_status on damage (Update_damage, Code/Body.h:2667-2700) with bonded contacts
        # (BondedMohrCoulomb after INITIALIZE_CZM, whose internal[0] the damage averages): two
        # entries evaluate the damage of loaded discs and never hold; a free rigid disc flying beside
        # the lattice (body 11, no contact: damage 1) turns inactive at the first update
        sc.laws = [(m1, m2, 5, 0, list(LAW_PARAMS[5])) for (m1, m2, _, _, _) in sc.laws]
        sc.initialize_czm = True
        xmax = max(b.nodes[:, 0].max() for b in sc.bodies)
        ymid = 0.5 * (min(b.nodes[:, 1].min() for b in sc.bodies) + max(b.nodes[:, 1].max() for b in sc.bodies))
        h = 2.0 * np.pi * 0.8e-3 / 32
        sc.bodies.append(g.make_rigid_disc((xmax + 4e-3, ymid), 0.8e-3, 32, 1, 7800.0, 0.5 * h, 0.5 * h,
                                           velocity=(0.01, 0.0)))
        sc.deactivation = ["Damage 0 above 2", "Damage 4 below 0.5", "Damage 11 above 0.99"]
    elif name in ("alid", "update_matrices"):
        # ALID absorbing layers on every grain: layers 0.9 mm wide along the lattice's outline,
        # graded quadratically, reference velocities of the layer in x and y; the stiffness
        # matrices (MATRICES, no damping) give the layers' coupling terms.  update_matrices: the
        # file's matrices come from half the grains' modulus and carry no damping, and
        # UPDATE_MASS/STIFFNESS/DAMPING_MATRIX rebuild masses, stiffness and Rayleigh damping
        # from the material (Body::Update_material), whose alpha and beta are set
        E, nu = (1e8, 0.3) if name == "alid" else (0.5e8, 0.3)
        g.add_damping(sc, 0.0, 0.0, E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu)))
        if name == "update_matrices":
            sc.update_matrices = (True, True, True)
            sc.materials = [(n, t, [p[0], 0.02 * sc.dt, 0.05 / sc.dt] + list(p[3:])) if n == "Grain" else (n, t, p)
                            for (n, t, p) in sc.materials]
        grains = [b for b in sc.bodies if b.kind == "deformable"]
        x0 = min(b.nodes[:, 0].min() for b in grains); x1 = max(b.nodes[:, 0].max() for b in grains)
        y0 = min(b.nodes[:, 1].min() for b in grains); y1 = max(b.nodes[:, 1].max() for b in grains)
        for b in grains:
            b.alid = {"x_hist": [(0.0, 0.0), (2e-5, 0.02), (g.T_HIST_END, 0.02)], "y_hist": [(0.0, -0.01), (g.T_HIST_END, -0.01)],
                      "xmin": x0, "xmax": x1, "ymin": y0, "ymax": y1, "range": 0.9e-3, "alphain": 0.0,
                      "alphaout": 0.05 * sc.dt, "betain": 0.0, "betaout": 0.1 / sc.dt, "exponent": 2.0}
    elif name == "neohookean":
        sc.materials = [(n, 1 if n == "Grain" else t, p) for (n, t, p) in sc.materials]
    elif name == "border_conditions":
        hist = lambda v: (np.array([0.0, g.T_HIST_END]), np.array([v, v]))
        combos = [((g.BC_SOFT, (1e8, 1e2), hist(0.02)), (g.BC_ORIENTED, (0.0, 0.0), hist(-2e4))),
                  ((g.BC_FOLLOWING, (0.0, 0.0), hist(3e4)), (g.BC_SOFT, (5e7, 0.0), hist(-0.01))),
                  ((g.BC_ORIENTED, (0.0, 0.0), hist(1e4)), (g.BC_FOLLOWING, (0.0, 0.0), hist(-1e4)))]
        for body, c in zip(sc.bodies[:3], combos):
            body.borders[0]["bc"] = list(c)
    return sc


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


CONTACT_KEYS = ["bodyS", "borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM", "nb_internal",
                "shapeM1", "shapeM2", "gapn", "vgapn", "gapt", "vgapt", "xsi", "xnorm", "ynorm", "fx", "fy",
                "internal0", "internal1", "internal2"]


def summary(node, contacts, works, pressures=None):
    """Digests of one state: node fields (name -> (n, 2) array), contacts (key -> column), works,
    border contact pressures ((n_border_nodes, 2): x, y)."""
    out = {"node_" + k: sha(v) for k, v in node.items()}
    if pressures is not None:
        out["contact_pressures"] = sha(pressures)
    out["n_contacts"] = int(len(contacts["fx"]))
    for k in CONTACT_KEYS:
        out["contact_" + k] = sha(contacts[k])
    out["works"] = sha(works)
    return out


def oracle_columns(c):
    """The oracle's contact records as the reference dump's columns."""
    cols = {k: c[k] for k in ("bodyS", "borderS", "border_nodeS", "nodeS", "bodyM", "borderM", "shiftM", "segmentM",
                              "nb_internal", "gapn", "vgapn", "gapt", "vgapt", "xsi", "xnorm", "ynorm", "fx", "fy")}
    for i in range(3):
        cols[f"internal{i}"] = c["internal"][:, i]
    cols["shapeM1"] = c["shapeM"][:, 1]
    cols["shapeM2"] = c["shapeM"][:, 2]
    return cols


def oracle_summary(o):
    st = o.node_state()
    f = o.forces()
    node = {"x": o.positions(), "up": st[:, 6:8], "f_int": f["internal"], "f_contact": f["contact"]}
    return summary(node, oracle_columns(o.contacts()), o.works(), o.contact_pressures())


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_per_case(oracle_built, case):
    from melody2d_b200 import generator as g
    from oracle.pyoracle import Oracle
    gold = json.load(open(GOLDEN))["cases"][case]
    flat = g.flatten(case_scene(case))
    assert input_checksum(flat) == gold["input_sha256"], "generated input differs from the fixture's input"
    o = Oracle(flat, correctly_rounded=False)
    done = 0
    for step in STEPS:
        o.step(step - done)
        done = step
        ref, got = gold["steps"][str(step)], oracle_summary(o)
        assert got["n_contacts"] == ref["n_contacts"], (case, step)
        assert ref["n_contacts"] > 0
        for k, v in ref.items():
            assert got[k] == v, f"{case}: {k} differs from the reference at step {step}"
