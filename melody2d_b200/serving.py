"""Serving loop for biaxial requests: continuous batching over the batch API (mel_batch_*).

Requests arrive as a seeded Poisson stream.  Each request is one biaxial sample of the batched
workload's distribution (grains log-uniform in [50,1000], 32-96 border nodes per grain,
confinement 50-400 kPa, friction 0.1-0.5) run until 5 % axial strain or a step cap.  The server:
  - builds each arriving request's model in a spawn process pool (the disc templates are built
    once per worker; the arrays come back in shared memory) and creates its solver in a thread
    pool (mel_create releases the GIL), after which the shared memory is freed;
  - admits created solvers into the resident batch while the estimated device memory of the
    residents stays within the HBM budget;
  - advances the batch in slices of one proximity period (10 steps), retiring each member when it
    reaches its stop criterion, and reads its monitored quantities back;
  - reports per-request latency (arrival to retirement), p50/p99, and completed samples per hour.
The same request stream can be served by the plain path: FP64 solvers run one at a time, in order
of arrival.  Both arms keep accepting arrivals while they compute."""
from __future__ import annotations

import dataclasses
import math
import multiprocessing as mp
import time
from concurrent.futures import ProcessPoolExecutor, ThreadPoolExecutor
from typing import Dict, List, Optional

import numpy as np

SLICE = 10                       # steps per batch call: one proximity period of the workload


@dataclasses.dataclass
class Request:
    rid: int
    seed: int
    arrival: float               # seconds after the start of the run
    target_steps: int = 0
    nodes: int = 0
    est_bytes: float = 0.0
    admitted: float = -1.0
    done: float = -1.0
    steps: int = 0
    kinetic_energy: float = 0.0
    wall_force: Optional[List[float]] = None
    failed: str = ""             # why the run stopped early (diverged state), empty when it completed
    shared: object = None        # the model's arrays in shared memory until its solver exists


def poisson_arrivals(rate: float, duration: float, seed: int) -> List[float]:
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def stop_steps(meta: dict, dt: float, strain: float, cap: int) -> int:
    """Steps to `strain` axial strain (the plates close at 2 v_plate on a sample of height H), or
    `cap`, rounded up to whole slices so that every arm runs a request for the same steps."""
    H = meta["box"][1]
    t = strain * H / (2.0 * meta["v_plate"])
    n = min(cap, math.ceil(t / dt))
    return int(math.ceil(n / SLICE) * SLICE)


# ---- request model building (spawn workers) -------------------------------------------------
_templates = None


def _init_worker(counts):
    global _templates
    from melody2d_b200 import generator as g
    _templates = g.DiscTemplates(counts, workers=1)


def _build(seed: int):
    """Worker: one request's model, its arrays handed over in shared memory (a model is hundreds
    of MB; through a pipe its transfer would cost more than its generation)."""
    from melody2d_b200 import generator as g
    sc = g.batch_sample_scene(seed, _templates)
    return seed, g.share_flat(g.flatten(sc)), sc.meta, sc.dt


def estimate_device_bytes(flat: dict) -> float:
    """Device memory of a solver created from `flat`: its arrays plus the chunk images, contact and
    proximity buffers (about 1.6x the description's arrays for these samples)."""
    host = sum(np.asarray(v).nbytes for k, v in flat.items() if k != "material_names")
    return 1.6 * host


class Server:
    def __init__(self, batched: bool = True, precision: int = 1, device: int = 0, hbm_budget: float = 150e9,
                 strain: float = 0.05, step_cap: int = 40000, build_workers: int = 8, create_threads: int = 4,
                 min_batch: int = 1):
        """min_batch: the batched arm holds admission until that many requests are ready (or no
        more are on their way), a batching window that trades first-request latency for fuller
        launches."""
        self.min_batch = min_batch
        self.batched, self.precision, self.device = batched, precision, device
        self.hbm_budget, self.strain, self.step_cap = hbm_budget, strain, step_cap
        self.build_workers, self.create_threads = build_workers, create_threads

    def run(self, arrivals: List[float], seeds: List[int], duration: float, drain: float = 0.0) -> Dict:
        from melody2d_b200.solver import Batch, MelError, Solver
        from melody2d_b200.abi import MEL_ERR_NAN, MEL_ERR_BOUNDS
        from melody2d_b200.generator import SharedFlat
        reqs = [Request(i, s, a) for i, (a, s) in enumerate(zip(arrivals, seeds))]
        ctx = mp.get_context("spawn")
        pool = ProcessPoolExecutor(max_workers=self.build_workers, mp_context=ctx, initializer=_init_worker,
                                   initargs=(list(range(32, 97)),))
        creators = ThreadPoolExecutor(max_workers=self.create_threads)
        batch = Batch(precision=self.precision, device=self.device) if self.batched else None
        building, creating = {}, {}
        ready: List = []                      # (request, solver) created, waiting for admission
        resident: Dict[int, tuple] = {}       # rid -> (request, solver)
        resident_bytes = 0.0
        nxt = 0
        t0 = time.perf_counter()
        gpu_ms = 0.0
        launches = 0
        max_resident = 0
        try:
            while True:
                now = time.perf_counter() - t0
                # arrivals within the run's window are accepted; the run ends after duration + drain
                while nxt < len(reqs) and reqs[nxt].arrival <= min(now, duration):
                    building[pool.submit(_build, reqs[nxt].seed)] = reqs[nxt]
                    nxt += 1
                for f in [f for f in building if f.done()]:
                    r = building.pop(f)
                    _, desc, meta, dt = f.result()
                    r.shared = SharedFlat(desc)
                    flat = r.shared.flat
                    r.target_steps = stop_steps(meta, dt, self.strain, self.step_cap)
                    ptr = np.asarray(flat["body_node_ptr"])
                    r.nodes = int(np.sum(np.diff(ptr)[np.asarray(flat["body_type"]) == 0]))
                    r.est_bytes = estimate_device_bytes(flat)
                    creating[creators.submit(Solver.from_flat, flat, self.precision, self.device, False)] = r
                for f in [f for f in creating if f.done()]:
                    r = creating.pop(f)
                    r.shared.release()
                    r.shared = None
                    ready.append((r, f.result()))
                ready.sort(key=lambda x: x[0].arrival)
                # admission: the batched arm takes every ready request that fits the budget; the plain
                # arm runs one request at a time
                more_coming = nxt < len(reqs) or building or creating
                hold = self.batched and not resident and len(ready) < self.min_batch and more_coming
                while ready and not hold and (self.batched or not resident):
                    r, s = ready[0]
                    if self.batched and resident and resident_bytes + r.est_bytes > self.hbm_budget:
                        break
                    ready.pop(0)
                    if self.batched:
                        batch.admit(s)
                    resident[r.rid] = (r, s)
                    resident_bytes += r.est_bytes
                    r.admitted = time.perf_counter() - t0
                max_resident = max(max_resident, len(resident))
                if resident:
                    failed = []
                    if self.batched:
                        failed = batch.step(SLICE)
                        st = batch.stats()
                        gpu_ms += st["ms_last_call"]
                        launches += st["launches"]
                    else:
                        (r, s), = resident.values()
                        try:
                            s.step(SLICE)
                        except MelError as e:
                            if e.code not in (MEL_ERR_NAN, MEL_ERR_BOUNDS):
                                raise
                            failed = [s]
                        gpu_ms += s.step_stats()["ms_total"]
                        launches += s.kernel_times()["launches"]
                    for rid in list(resident):
                        r, s = resident[rid]
                        if s in failed:                  # the sample diverged: it stops here
                            r.failed = s.health()[1] if self.batched else "diverged"
                            s.close()
                            del resident[rid]
                            resident_bytes -= r.est_bytes
                            r.done = time.perf_counter() - t0
                            continue
                        r.steps += SLICE
                        if r.steps >= r.target_steps:
                            if self.batched:
                                batch.retire(s)
                            m = s.monitor()
                            r.kinetic_energy = m.kinetic_energy
                            r.wall_force = list(m.rigid_force)
                            s.close()
                            del resident[rid]
                            resident_bytes -= r.est_bytes
                            r.done = time.perf_counter() - t0
                else:
                    time.sleep(0.002)
                now = time.perf_counter() - t0
                if now >= duration + drain or (now >= duration and nxt == len(reqs) and not building
                                               and not creating and not ready and not resident):
                    break
        finally:
            for r, s in list(resident.values()):
                s.close()
            for r, s in ready:
                s.close()
            if batch is not None:
                batch.close()
            creators.shutdown(wait=True, cancel_futures=True)
            for f, r in creating.items():
                if f.done() and not f.cancelled() and not f.exception():
                    f.result().close()
                if r.shared is not None:
                    r.shared.release()
            for f in building:
                f.cancel()
            for f in building:               # models already being built: wait, then free them
                try:
                    SharedFlat(f.result()[1]).release()
                except BaseException:
                    pass
            pool.shutdown(wait=False, cancel_futures=True)
        wall = time.perf_counter() - t0
        failed = [r for r in reqs if r.done >= 0 and r.failed]
        done = [r for r in reqs if r.done >= 0 and not r.failed]
        lat = np.array([r.done - r.arrival for r in done])
        arrived = [r for r in reqs if r.arrival <= duration]
        return {
            "arm": "batched" if self.batched else "plain",
            "precision": "mixed" if self.precision == 1 else "fp64",
            "arrived": len(arrived), "completed": len(done), "failed": len(failed),
            "in_flight_at_end": len(arrived) - len(done) - len(failed),
            "wall_s": wall, "samples_per_hour": len(done) * 3600.0 / wall,
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_steps": float(np.mean([r.target_steps for r in done])) if done else None,
            "mean_nodes": float(np.mean([r.nodes for r in done])) if done else None,
            "gpu_ms": gpu_ms, "gpu_launches": launches, "max_resident": max_resident,
            "requests": [{"rid": r.rid, "seed": r.seed, "arrival": r.arrival, "admitted": r.admitted, "done": r.done,
                          "steps": r.target_steps, "nodes": r.nodes, "kinetic_energy": r.kinetic_energy,
                          "wall_force": r.wall_force} for r in done],
        }
