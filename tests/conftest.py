"""Shared fixtures.  Tests marked `gpu` need a CUDA device and libmelgpu.so; everything else runs
on the CPU (oracle, generator, loader, ABI symbol checks)."""
import functools
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmelgpu.so")


@functools.lru_cache(maxsize=None)
def squeezed_lattice(nx=4, ny=4, seed=0, nsteps=300):
    """Config-0 geometry with a 2.05 mm pitch and plates starting 1 um inside the outer discs, so
    disc-disc and disc-plate contacts carry force from the first step."""
    from melody2d_b200 import generator as g
    return g.disc_lattice_scene(seed=seed, nx=nx, ny=ny, pitch=2.05e-3, gap0=-1e-6, nsteps=nsteps)


def outputs_scene(nsteps=60):
    """A 2x2 squeezed lattice of small discs with a MONITORING list covering every entry type the
    device monitoring computes, MONITOR_ENERGY, and saves every 30 steps: the case of the
    reference-format output tests (fixtures written by tests/golden/make_golden_outputs.py)."""
    from melody2d_b200 import generator as g
    sc = g.disc_lattice_scene(seed=5, nx=2, ny=2, pitch=2.05e-3, gap0=-1e-6, nsteps=nsteps, n_border=24,
                              n_interior=24, min_sep=0.15e-3, name="outputs")
    n = [b.nodes.shape[0] for b in sc.bodies]
    # a whole-body force entry sums as many nodes as body number <force kind> has (the reference's
    # loop bound): Contact (kind 2) on the disc with the most nodes stays inside it
    big = max(range(4), key=lambda b: n[b])
    assert n[big] >= n[2]
    sc.monitored = ["Position Y 4 -1", "Position X 0 -1", "Position Y 1 7", "Displacement Mag 1 5",
                    "Displacement R 5 -1", "Velocity Y 5 -1", "Velocity X 3 -1", "Acceleration X 2 -1",
                    "Acceleration Mag 4 -1", "Force Y Contact 4 -1", "Force X Total 0 3",
                    "Force Mag Internal 1 2", "Force X Body 2 4", "Force Y Dirichlet 5 -1",
                    "Force X Contact %d -1" % big, "Force Y Neumann 0 1", "Contact Gapn 0 0 7",
                    "Contact Xnorm 1 0 3", "Energy Kinetic 0", "Energy Kinetic 4", "Energy Kinetic -1",
                    "Energy Deformation 1", "Work Contact 0", "Work Dirichlet -1", "Work Internal 5",
                    "Error X 0 1", "Position AllX"]
    sc.monitor_energy = True
    sc.save_period = 30 * sc.dt
    sc.print_period = 20 * sc.dt
    return sc


_FLAT = {}


def flat_of(scene):
    from melody2d_b200 import generator as g
    key = id(scene)
    if key not in _FLAT:
        _FLAT[key] = (scene, g.flatten(scene))
    return _FLAT[key][1]


def input_checksum(flat) -> str:
    import hashlib
    h = hashlib.sha256()
    for k in sorted(flat):
        if k == "material_names":
            continue
        if k == "deactivated" and np.asarray(flat[k]).size == 0:
            continue                      # models without DEACTIVATION hash as before the field existed
        h.update(k.encode())
        h.update(np.ascontiguousarray(np.asarray(flat[k])).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="session")
def oracle_built():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    return True


@pytest.fixture(scope="session")
def gpu_lib():
    """libmelgpu.so; GPU tests fail loudly (no fallback) when it cannot be built or loaded."""
    from melody2d_b200 import build, solver
    build.build()
    return solver.lib()
