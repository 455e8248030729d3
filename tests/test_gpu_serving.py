"""Serving loop (melody2d_b200/serving.py): requests that arrive while others are on the GPU are
admitted into the resident batch, and each request's result is the same alone and in the mix --
bit for bit, since a batch member computes what it would alone -- and within the mixed form's
tolerance (1e-5 relative) of the plain FP64 path serving one request at a time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_match_alone_and_plain(gpu_lib):
    from melody2d_b200 import generator as g
    from melody2d_b200.serving import Server, stop_steps
    from melody2d_b200.solver import Solver
    arrivals = [0.0, 0.05, 0.1, 0.6, 0.65, 1.2]
    seeds = [900 + i for i in range(len(arrivals))]
    # a batching window of all six requests makes them share the GPU whatever the build times
    batched = Server(batched=True, precision=1, step_cap=150, build_workers=3, create_threads=2,
                     min_batch=len(arrivals)).run(arrivals, seeds, duration=2.0, drain=120.0)
    assert batched["completed"] == len(arrivals)
    assert batched["max_resident"] == len(arrivals)
    rows = {r["seed"]: r for r in batched["requests"]}
    templates = g.DiscTemplates(range(32, 97), workers=1)
    for seed in seeds:
        sc = g.batch_sample_scene(seed, templates)
        assert rows[seed]["steps"] == stop_steps(sc.meta, sc.dt, 0.05, 150)
        s = Solver.from_flat(g.flatten(sc), precision=1)
        s.step(rows[seed]["steps"])
        m = s.monitor()
        assert m.kinetic_energy == rows[seed]["kinetic_energy"]
        assert list(m.rigid_force) == rows[seed]["wall_force"]
        s.close()
    plain = Server(batched=False, precision=0, step_cap=150, build_workers=3, create_threads=2).run(
        arrivals, seeds, duration=2.0, drain=120.0)
    assert plain["completed"] == len(arrivals)
    for r in plain["requests"]:
        b = rows[r["seed"]]
        assert abs(b["kinetic_energy"] - r["kinetic_energy"]) <= 1e-5 * abs(r["kinetic_energy"])
        wb, wp = np.array(b["wall_force"]), np.array(r["wall_force"])
        assert np.linalg.norm(wb - wp) <= 1e-5 * max(np.linalg.norm(wp), 1e-300)
