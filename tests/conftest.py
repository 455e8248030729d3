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
