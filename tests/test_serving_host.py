"""The serving loop's host logic on the CPU, with stand-ins for the GPU solver and batch: every
request of a Poisson stream is built (spawn workers, model arrays handed over in shared memory),
created, admitted, advanced and retired at its stop step, latencies are reported, and no
shared-memory block outlives the run."""
import os
import types

import pytest


class _FakeSolver:
    created = 0

    def __init__(self, flat):
        self.nodes = len(flat["node_domain"])
        self.steps = 0
        _FakeSolver.created += 1

    @classmethod
    def from_flat(cls, flat, precision=0, device=0, retain=True):
        assert not retain, "the serving loop must not keep the shared arrays"
        return cls(flat)

    def step(self, n=1):
        self.steps += n

    def step_stats(self):
        return {"ms_total": 0.01 * self.steps}

    def kernel_times(self):
        return {"launches": 3 * self.steps}

    def monitor(self):
        return types.SimpleNamespace(kinetic_energy=float(self.steps), rigid_force=[0.0] * 12)

    def health(self):
        return 0, ""

    def close(self):
        pass


class _FakeBatch:
    def __init__(self, precision=0, device=0):
        self.members = []

    def admit(self, s):
        self.members.append(s)

    def retire(self, s):
        self.members.remove(s)

    def step(self, n=1, proximity=True):
        for s in self.members:
            s.step(n)
        return []

    def stats(self):
        return {"ms_last_call": 1.0, "launches": 3, "members": len(self.members)}

    def close(self):
        self.members = []


def _shm_blocks():
    return {f for f in os.listdir("/dev/shm") if f.startswith("psm_")} if os.path.isdir("/dev/shm") else set()


@pytest.mark.parametrize("batched", [True, False])
def test_serving_loop_host_logic(monkeypatch, batched):
    import melody2d_b200.solver as solver
    from melody2d_b200.serving import Server, SLICE
    monkeypatch.setattr(solver, "Solver", _FakeSolver)
    monkeypatch.setattr(solver, "Batch", _FakeBatch)
    before = _shm_blocks()
    arrivals, seeds = [0.05, 0.1, 0.3], [21, 22, 23]
    srv = Server(batched=batched, precision=1 if batched else 0, hbm_budget=150e9, strain=0.05, step_cap=3 * SLICE,
                 build_workers=2, create_threads=2, min_batch=1)
    out = srv.run(arrivals, seeds, duration=1.0, drain=120.0)
    assert out["completed"] == 3 and out["failed"] == 0 and out["in_flight_at_end"] == 0
    assert all(r["steps"] == 3 * SLICE for r in out["requests"])
    assert all(r["kinetic_energy"] == 3 * SLICE for r in out["requests"])
    assert out["latency_p50_s"] is not None and out["latency_p99_s"] >= out["latency_p50_s"]
    assert _shm_blocks() <= before
