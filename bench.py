"""Throughput of the MELODY 2D explicit step on B200: node-steps/s on the 2000-disc biaxial sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--discs 2000]

One JSON line on rank 0.  A step is one Euler_step (Code/Solver.h:10-88) of the whole sample plus
the proximity updates that fall in it (Code/main.cpp:191-196, every 10 steps).  `value` is deformable
node-steps per second of device time over the timed K steps (inputs ~1.7 GB per step, larger than
L2).  `e2e` repeats the measurement through the public C ABI with the state in host memory, as the
reference keeps it: every step uploads the node state from a pinned host buffer, steps, downloads the
node state and reads the monitored quantities.  `cpu_baseline` is the reference solver, compiled from
its sources, timed on this host's cores on a bounded sample of the same workload.  At N=1 the line
also carries the headline of the batched and serving forms: `batched` (a slice of the batched
workload, mixed precision in one batch, against the plain FP64 path one sample at a time) and
`serving` (a short Poisson request stream served by continuous batching, p50/p99 latency).  Under
torchrun every rank advances its own independent sample (weak scaling, no collective in the step).
`--impl reference` times the reference itself on the same 2000-disc sample."""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s"
DEFAULT_STEPS = 2000
DEFAULT_WARMUP = 20


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() in ("active", "1", "yes")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def allreduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


# --------------------------------------------------------------------------------------------
# reference CPU path (the reference solver compiled from its sources, oracle/_ref)
# --------------------------------------------------------------------------------------------
def reference_sample(n_discs: int, steps: int, threads: int, seed: int = 1):
    """Runs the reference's own Euler_step loop (oracle/_ref/ref_harness) on a seeded sample of the
    biaxial workload (same disc size distribution, nodes per disc, materials, contact law, loading;
    seed 1 and 2000 discs is the sample the GPU arm times) and returns node-steps/s of its step
    loop (wall clock of the loop alone, after Load_static, Load_dynamic and the set-up)."""
    from melody2d_b200 import generator as g
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    scene = g.biaxial_scene(seed=seed, n_discs=n_discs, workers=threads)
    with tempfile.TemporaryDirectory() as tmp:
        g.write_asc(scene, tmp, workers=threads)
        if os.path.exists(harness):
            out = subprocess.run([harness, tmp, str(steps), "-", "0", str(threads)], check=True,
                                 capture_output=True, text=True).stdout
            r = json.loads(out.strip().splitlines()[-1])
            return r["deformable_nodes"] * r["steps"] / r["wall_s"], threads, "reference", scene
    # no compiled reference on this machine: the C restatement (one thread)
    from oracle.pyoracle import Oracle
    flat = g.flatten(scene)
    o = Oracle(flat)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return scene.n_deformable_nodes * steps / dt, 1, "port", scene


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def workload_name(discs: int) -> str:
    return (f"biaxial: {discs} deformable discs, radii U[0.5,1.5] mm, 64 border + 340 interior nodes each, MLS "
            f"(linear, W1), ElasticLinear, MohrCoulomb, mass x100, plates 0.05 m/s, walls 100 kPa; Euler, "
            f"dt=0.5 dt_crit; proximity every 10 steps")


def run_reference(args, rank, world, pg):
    """The reference solver alone, on the sample the GPU arm times (seed 1, args.discs discs), for
    args.ref_arm_steps steps of its own loop on all host threads; only rank 0 works."""
    if rank != 0:
        return
    threads = host_threads()
    steps = args.ref_arm_steps
    rate, cores, kind, scene = reference_sample(args.discs, steps, threads, seed=1)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "node-steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": 0, "ms_per_step": 1e3 * scene.n_deformable_nodes / rate,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded biaxial packing generator)",
            "config": {"workload": workload_name(args.discs), "nodes_per_gpu": scene.n_deformable_nodes,
                       "precision": "fp64", "sample": f"the GPU arm's sample (seed 1), the first {steps} steps "
                                                    f"of its loop timed after set-up"},
            "cpu_baseline": {"value": rate, "unit": "node-steps/s", "cores": cores, "kind": kind,
                             "sample": f"the full {args.discs}-disc sample, {steps} steps, all host threads"},
            "e2e": {"value": rate, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------------
# our path
# --------------------------------------------------------------------------------------------
def run_ours(args, rank, world, local, pg):
    import ctypes
    from melody2d_b200 import abi, generator as g
    from melody2d_b200.solver import PinnedArray, Solver, lib as solver_lib
    workers = max(1, host_threads() // max(1, world))
    t0 = time.perf_counter()
    scene = g.biaxial_scene(seed=1 + rank, n_discs=args.discs, workers=workers)
    flat = g.flatten(scene)
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    precision = 1 if args.precision == "mixed" else 0
    s = Solver.from_flat(flat, precision=precision, device=local)
    t_create = time.perf_counter() - t0
    model_bytes = sum(np.asarray(v).nbytes for k, v in flat.items() if k != "material_names")
    nodes = s.step_stats()["n_deformable_nodes"]
    s.step(args.warmup)
    s.set_timing(True)
    clocks = ClockSampler(local)
    barrier(pg)
    clocks.start()
    io_t = s.step(args.steps)                             # synchronises on its stream at the end
    barrier(pg)
    clk = clocks.stop()
    st = s.step_stats()
    kt = s.kernel_times()
    ms_total = allreduce_max(pg, st["ms_total"])
    value = allreduce_sum(pg, nodes) * args.steps / (ms_total * 1e-3)
    # roofline of the dominant kernel (body kernel), from its CUDA-event time in the region
    body_ms = kt["body"] / args.steps
    contact_ms = kt["contact"] / args.steps
    peak, peak_kind = measured_hbm_peak()
    achieved = st["bytes_body"] / (body_ms * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "body_kernel_traffic.json")
    if os.path.exists(prof):
        try:
            per_gp = json.load(open(prof))["dram_bytes_per_gauss_point"].get(args.precision)
            traffic = per_gp * s.sizes()["n_gauss"] if per_gp else None
        except Exception:
            traffic = None
    # end to end through the C ABI with the state in host memory (where the reference keeps it):
    # every iteration uploads the node state from a pinned host buffer, steps once, downloads the
    # node state and reads the monitored quantities back
    s.set_timing(False)
    n_e2e = min(args.steps, args.e2e_steps)
    L = solver_lib()
    host = PinnedArray(12 * s.nn)
    hp = host.array.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    mon = abi.MelMonitor()
    io = abi.MelStepIO(nsteps=1, run_proximity=1)
    L.mel_get_node_state(s.h, hp)
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        rc = L.mel_set_node_state(s.h, hp) or L.mel_step(s.h, ctypes.byref(io)) or \
            L.mel_get_node_state(s.h, hp) or L.mel_monitor_compute(s.h, ctypes.byref(mon))
        if rc:
            raise RuntimeError(L.mel_last_error_string().decode())
    t_e2e = time.perf_counter() - t0
    t_e2e = allreduce_max(pg, t_e2e)
    host.close()
    e2e_value = allreduce_sum(pg, nodes) * n_e2e / t_e2e
    # the same loop with the state left on the device (only the monitored quantities come back)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        s.step(1)
        s.monitor()
    t_res = allreduce_max(pg, time.perf_counter() - t0)
    resident_value = allreduce_sum(pg, nodes) * n_e2e / t_res
    n_solver_nodes = s.nn
    sizes = s.sizes()
    s.close()
    extras = {}
    if world == 1 and not args.no_extras:
        extras = headline_extras(args, rank, world, local, pg)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rate, cores, kind, _ = reference_sample(args.ref_discs, args.ref_steps, host_threads())
        cpu = {"value": rate, "unit": "node-steps/s", "cores": cores, "kind": kind,
               "sample": f"{args.ref_discs}-disc sample of the same workload, {args.ref_steps} steps, all host threads"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "node-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if precision == 0 else "f32 (dN, strain, stress, contributions) + f64",
            "data": "synthetic (seeded biaxial packing generator)",
            "config": {"workload": workload_name(args.discs), "nodes_per_gpu": nodes, "gauss_points": sizes["n_gauss"], "gp_entries": sizes["n_gp_entries"],
                       "contacts": st["n_contacts"], "precision": args.precision,
                       "l2": "inputs larger than L2 (%.2f GB streamed per step)" % ((st["bytes_body"] + st["bytes_contact"]) / 1e9),
                       "generate_s": round(t_gen, 2), "create_s": round(t_create, 2)},
            "e2e": {"value": e2e_value, "unit": "node-steps/s", "h2d_bytes_per_step": 96 * n_solver_nodes,
                    "d2h_bytes_per_step": 96 * n_solver_nodes + ctypes.sizeof(abi.MelMonitor), "steps": n_e2e,
                    "calls": "per step: mel_set_node_state (pinned host buffer), mel_step(nsteps=1), "
                             "mel_get_node_state (pinned host buffer), mel_monitor_compute; host wall clock",
                    "inputs": "the node state (12 doubles per node: u, v, a and their parameters) lives in host "
                              "memory as in the reference and crosses the host link both ways every step; the "
                              "model itself is uploaded once by mel_create (setup.h2d_bytes)",
                    "resident_state": {"value": resident_value, "calls": "mel_step(nsteps=1) then "
                                       "mel_monitor_compute, state kept on the device"},
                    "setup": {"h2d_bytes": int(model_bytes), "create_s": round(t_create, 2)}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "kernel": "body_kernel", "peak_source": peak_kind,
                         "bytes_per_launch": st["bytes_body"], "ms_per_launch": body_ms,
                         "contact_kernel_ms": contact_ms, "proximity_ms_per_step": kt["proximity"] / args.steps},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": kt["launches"],
            "proximity_updates": io_t.n_proximity,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)


def headline_extras(args, rank, world, local, pg):
    """The batched and serving figures beside the single-sample line (one GPU): a slice of the batched
    workload in one mixed-precision batch against the plain FP64 path one sample at a time (samples
    per hour extrapolated to the workload's 20,000 steps per sample, and the mixed form's errors),
    and a short serving run (p50/p99 latency, samples per hour of both arms)."""
    import copy
    out = {}
    a = copy.copy(args)
    a.samples, a.plain_subset = args.batch_samples, args.batch_plain_subset
    a.accuracy_samples, a.accuracy_steps = args.batch_accuracy_samples, args.batch_accuracy_steps
    a.steps, a.warmup = max(args.steps, 20), max(args.warmup, 3)
    b = run_batch(a, rank, world, local, pg, emit=False)
    if b is not None:
        out["batched"] = {"metric": "samples/h", "value": b["value"], "unit": "samples/h",
                          "ms_per_step": b["ms_per_step"], "steps": a.steps, "node_steps_per_s": b["node_steps_per_s"],
                          "config": b["config"], "plain_fp64_one_at_a_time": b["plain_fp64_one_at_a_time"],
                          "ratio_vs_plain_fp64": b["ratio_vs_plain_fp64"], "accuracy_vs_fp64": b["accuracy_vs_fp64"],
                          "gpu_launches": b["gpu_launches"], "clocks": b["clocks"]}
    try:
        out["input_generation"] = input_generation(args, local)
    except Exception as e:                       # reported, never silently dropped
        out["input_generation"] = {"error": str(e)}
    try:
        out["launch_overhead"] = launch_overhead(args, local)
    except Exception as e:
        out["launch_overhead"] = {"error": str(e)}
    a = copy.copy(args)
    a.rate, a.duration, a.drain, a.step_cap = args.serve_rate, args.serve_duration, args.serve_drain, args.serve_step_cap
    v = run_serve(a, rank, world, local, pg, emit=False)
    if v is not None:
        out["serving"] = {"metric": "samples/h", "value": v["value"], "unit": "samples/h", "config": v["config"],
                          "arms": v["arms"], "ratio_samples_h_vs_plain_fp64": v["ratio_samples_h_vs_plain_fp64"],
                          "same_requests_compared": v["same_requests_compared"],
                          "max_rel_error_vs_plain_fp64": v["max_rel_error_vs_plain_fp64"]}
    return out


def input_generation(args, local):
    """Gauss-point shape functions of a generated sample on the device (mel_mls_shapes) against
    the host restatement of the pre-processor's MLS pass (generator.mls_shape, one thread), in
    Gauss points per second; the device figure is the value pass's CUDA-event time, the e2e figure
    the whole call with its host transfers."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import mls_shapes
    sc = g.biaxial_scene(seed=11, n_discs=args.mls_discs, workers=host_threads())
    bodies = [b for b in sc.bodies if b.kind == "deformable"]
    jobs = [(b.gp_xy, b.nodes, b.domain) for b in bodies]
    npts = sum(j[0].shape[0] for j in jobs)
    mls_shapes(jobs[:8], device=local)                      # warm-up (module load, allocations)
    best_k, best_w, entries = None, None, 0
    for _ in range(3):
        tm = {}
        t0 = time.perf_counter()
        out = mls_shapes(jobs, device=local, timing=tm)
        w = time.perf_counter() - t0
        best_k = tm["kernel_ms"] if best_k is None else min(best_k, tm["kernel_ms"])
        best_w = w if best_w is None else min(best_w, w)
        entries = sum(len(o[1]) for o in out)
    sub = jobs[:args.mls_cpu_bodies]
    t0 = time.perf_counter()
    for pts, nodes, radii in sub:
        g.mls_shape(pts, nodes, radii, np.zeros(2))
    cpu_s = time.perf_counter() - t0
    cpu_pts = sum(j[0].shape[0] for j in sub)
    written = entries * (4 + 3 * 8) + (npts + 1) * 8
    return {"metric": "Gauss points/s", "value": npts / (best_k * 1e-3), "unit": "points/s",
            "e2e": {"value": npts / best_w, "unit": "points/s"},
            "config": {"workload": "shape functions of the %d-disc biaxial sample" % args.mls_discs,
                       "gauss_points": npts, "support_entries": entries},
            "value_pass_ms": best_k, "bytes_written": written,
            "achieved_write_gbs": written / (best_k * 1e-3) / 1e9,
            "cpu_baseline": {"value": cpu_pts / cpu_s, "unit": "points/s", "cores": 1, "kind": "port",
                             "sample": "%d bodies (%d points) through generator.mls_shape" % (len(sub), cpu_pts)}}


def launch_overhead(args, local):
    """Evidence for the K-step CUDA graph question on the smallest workload, where launches weigh
    most: the 4x4 lattice (config 0, 2.4 k nodes) stepped 1000 times in one mel_step call.  Host wall
    clock, device time between the first and last launch (CUDA events), and the sum of the kernels'
    own times (events around each launch, a separate run); the gap between the last two is the time
    the GPU waits for launches, which a captured graph could remove."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    s = Solver.from_flat(g.flatten(g.disc_lattice_scene()), device=local)
    try:
        s.step(20)
        n = 1000
        t0 = time.perf_counter()
        s.step(n)
        wall = (time.perf_counter() - t0) * 1e3 / n
        st = s.step_stats()
        dev = st["ms_total"] / n
        launches = s.kernel_times()["launches"] / n
        s.set_timing(True)
        s.step(n)
        kt = s.kernel_times()
        kern = (kt["contact"] + kt["body"] + kt["proximity"]) / n
        return {"workload": "4x4 lattice, 2.4 k nodes, 1000 steps per mel_step call",
                "host_wall_ms_per_step": wall, "device_ms_per_step": dev, "kernel_ms_per_step": kern,
                "launches_per_step": launches, "gpu_waiting_fraction": max(0.0, 1.0 - kern / dev)}
    finally:
        s.close()


def create_solvers(flats, precision, device, threads):
    """mel_create for many samples at once (the library call releases the interpreter lock)."""
    from concurrent.futures import ThreadPoolExecutor
    from melody2d_b200.solver import Solver
    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(lambda f: Solver.from_flat(f, precision=precision, device=device, retain=False), flats))


def run_batch(args, rank, world, local, pg, emit=True):
    """Batched workload: S independent biaxial samples (grains log-uniform in [50,1000], 32-96
    border nodes per grain, confinement 50-400 kPa, friction 0.1-0.5) advanced together in one
    mixed-precision batch, against the plain FP64 path run one sample at a time on a subset.
    Samples/h are extrapolated from the timed steps to sample_steps steps per sample."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Batch, Solver
    threads = max(1, host_threads() // max(1, world))
    seeds = [1000 * (rank + 1) + i for i in range(args.samples)]
    # the plain FP64 subset; its samples stay mapped for the plain and accuracy legs
    sub = list(range(0, args.samples, max(1, args.samples // args.plain_subset)))[: args.plain_subset]
    t0 = time.perf_counter()
    # generation (spawn workers, samples handed over in shared memory) overlapped with mel_create
    solvers, kept, _ = g.build_batch_samples(
        seeds, lambda f: Solver.from_flat(f, precision=1, device=local, retain=False),
        workers=threads, create_threads=max(2, threads // 2), keep=sub)
    t_build = time.perf_counter() - t0
    flats = {i: sf.flat for i, sf in kept.items()}
    nodes = [s.step_stats()["n_deformable_nodes"] for s in solvers]
    b = Batch(precision=1, device=local)
    for s in solvers:
        b.admit(s)
    b.step(args.warmup)
    launches0 = b.stats()["launches"]
    clocks = ClockSampler(local)
    barrier(pg)
    clocks.start()
    b.step(args.steps)
    barrier(pg)
    clk = clocks.stop()
    st = b.stats()
    ms = allreduce_max(pg, st["ms_last_call"])
    total_nodes = allreduce_sum(pg, sum(nodes))
    value = total_nodes * args.steps / (ms * 1e-3)
    ms_per_step = ms / args.steps
    samples_h = allreduce_sum(pg, args.samples) * 3600.0 / (ms_per_step * 1e-3 * args.sample_steps)
    b.close()
    for s in solvers:
        s.close()
    # plain FP64 path, one sample at a time, on a subset
    plain_ms = []
    for i in sub:
        a = create_solvers([flats[i]], 0, local, 1)[0]
        a.step(args.warmup)
        a.step(args.steps)
        plain_ms.append(a.step_stats()["ms_total"] / args.steps)
        a.close()
    # the subset's mean time per step alone stands for the mean sample of the distribution
    plain_samples_h = 3600.0 / (float(np.mean(plain_ms)) * 1e-3 * args.sample_steps)
    # accuracy of the mixed form against the FP64 path after args.accuracy_steps steps (grains and
    # walls in contact by then), on the first samples of the subset; a batch member's state equals
    # the same sample stepped alone, so the samples run alone here
    errs = []
    for i in sub[: args.accuracy_samples]:
        a = create_solvers([flats[i]], 0, local, 1)[0]
        m = create_solvers([flats[i]], 1, local, 1)[0]
        a.step(args.accuracy_steps)
        m.step(args.accuracy_steps)
        ma, mb = a.monitor(), m.monitor()

        def rel(x, y):
            x, y = np.asarray(x, float), np.asarray(y, float)
            return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        errs.append({"kinetic_energy": rel(mb.kinetic_energy, ma.kinetic_energy),
                     "wall_contact_force": rel(list(mb.rigid_force), list(ma.rigid_force)),
                     "wall_reaction": rel(list(mb.rigid_dirichlet), list(ma.rigid_dirichlet)),
                     "active_contacts": [mb.active_contacts, ma.active_contacts]})
        a.close()
        m.close()
    if rank == 0:
        line = {
            "metric": "samples/h", "value": samples_h, "unit": "samples/h", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (dN, strain, stress, contributions) + f64",
            "data": "synthetic (seeded batched biaxial generator, scaled disc templates)",
            "config": {"workload": f"batched: {args.samples} independent biaxial samples per GPU, grains log-uniform "
                                   f"[50,1000], 32-96 border + 5x interior nodes per grain, confinement U[50,400] kPa, "
                                   f"friction U[0.1,0.5], mass x100, plates 0.05 m/s; mixed precision",
                       "samples_per_gpu": args.samples, "nodes_per_gpu": int(sum(nodes)),
                       "samples_h_extrapolated_to_steps": args.sample_steps,
                       "l2": "inputs larger than L2", "build_s": round(t_build, 2),
                       "build": "generation in spawn workers, samples handed over in shared memory, overlapped with mel_create"},
            "node_steps_per_s": value,
            "plain_fp64_one_at_a_time": {"samples_h": plain_samples_h, "subset": len(sub),
                                         "ms_per_step_mean": float(np.mean(plain_ms))},
            "ratio_vs_plain_fp64": samples_h / plain_samples_h if world == 1 else None,
            "accuracy_vs_fp64": {"steps": args.accuracy_steps, "samples": len(errs),
                                 "max_rel_error": {k: max(e[k] for e in errs) for k in ("kinetic_energy", "wall_contact_force", "wall_reaction")} if errs else None,
                                 "active_contacts_mixed_fp64": [e["active_contacts"] for e in errs]},
            "clocks": clk, "gpu_launches": st["launches"] - launches0,
        }
        if emit:
            print(json.dumps(line), flush=True)
    flats.clear()
    for sf in kept.values():
        sf.release()
    return line if rank == 0 else None


def run_serve(args, rank, world, local, pg, emit=True):
    """Serving: seeded Poisson arrivals (args.rate per second for args.duration seconds) of
    batched-workload requests, each run to 5 % axial strain or args.step_cap steps; the batched
    mixed-precision server against the plain FP64 path serving one request at a time, on the same
    request stream.  Both arms get args.drain seconds after the last arrival to finish."""
    from melody2d_b200.serving import Server, poisson_arrivals
    arrivals = poisson_arrivals(args.rate, args.duration, seed=7 + rank)
    seeds = [50000 * (rank + 1) + i for i in range(len(arrivals))]
    threads = max(1, host_threads() // max(1, world))
    arms = {}
    for name, batched, precision in (("batched_mixed", True, 1), ("plain_fp64", False, 0)):
        srv = Server(batched=batched, precision=precision, device=local, hbm_budget=args.hbm_budget * 1e9,
                     step_cap=args.step_cap, build_workers=max(1, threads - 6), create_threads=6)
        barrier(pg)
        res = srv.run(arrivals, seeds, args.duration, drain=args.drain)
        arms[name] = res
    # same request, both arms: the final monitored quantities agree within the mixed form's tolerance
    a = {r["rid"]: r for r in arms["batched_mixed"]["requests"]}
    b = {r["rid"]: r for r in arms["plain_fp64"]["requests"]}
    common = sorted(set(a) & set(b))

    def rel(x, y):
        x, y = np.asarray(x, float), np.asarray(y, float)
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    err_ke = max([rel(a[i]["kinetic_energy"], b[i]["kinetic_energy"]) for i in common], default=None)
    err_wall = max([rel(a[i]["wall_force"], b[i]["wall_force"]) for i in common], default=None)
    if rank == 0:
        summary = {k: {kk: v for kk, v in r.items() if kk != "requests"} for k, r in arms.items()}
        line = {
            "metric": "samples/h", "value": summary["batched_mixed"]["samples_per_hour"], "unit": "samples/h",
            "n_gpus": world, "steps": None, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (dN, strain, stress, contributions) + f64",
            "data": "synthetic (seeded Poisson request stream of batched-workload samples)",
            "config": {"workload": f"serving: Poisson arrivals at {args.rate}/s for {args.duration} s, requests from the "
                                   f"batched-workload distribution, each to 5% axial strain or {args.step_cap} steps, "
                                   f"HBM budget {args.hbm_budget} GB, {args.drain} s drain"},
            "arms": summary,
            "ratio_samples_h_vs_plain_fp64": (summary["batched_mixed"]["samples_per_hour"] /
                                              max(summary["plain_fp64"]["samples_per_hour"], 1e-300)),
            "same_requests_compared": len(common),
            "max_rel_error_vs_plain_fp64": {"kinetic_energy": err_ke, "wall_contact_force": err_wall},
            "gpu_launches": summary["batched_mixed"]["gpu_launches"],
        }
        if emit:
            print(json.dumps(line), flush=True)
        return line
    return None


def compare_precisions(args, rank, world, local, pg):
    """Config-2 report: the mixed form against the FP64 path (bit-identical to the FP64 oracle) on
    the same generated sample after K steps: relative errors of kinetic energy, wall reaction
    (contact force and driven-DOF reaction of the rigid plates and walls), mass-weighted mean
    displacement, and the two active-contact counts."""
    from melody2d_b200 import generator as g
    from melody2d_b200.solver import Solver
    if rank != 0:
        return
    scene = g.biaxial_scene(seed=1, n_discs=args.discs, workers=host_threads())
    flat = g.flatten(scene)
    a = Solver.from_flat(flat, precision=0, device=local)
    b = Solver.from_flat(flat, precision=1, device=local)
    # chaos gauge: an FP64 twin whose displacement parameters are moved by 1e-16 m (about 1e-12 of
    # the nodal spacing, a seeded pattern, so not a rigid translation) after 100 steps: how fast the
    # sample itself amplifies a difference, whatever its source.  (Most parameters are still exactly
    # zero then, so a one-ulp change would be a subnormal that the strain products round away.)
    c = Solver.from_flat(flat, precision=0, device=local)
    for sv in (a, b, c):
        sv.step(100)
    st = c.node_state()
    st[:, 6:8] += 1e-16 * np.random.default_rng(0).standard_normal(st[:, 6:8].shape)
    c.set_node_state(st)
    done0 = 100

    def rel(x, y):
        x, y = np.asarray(x, float), np.asarray(y, float)
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    from melody2d_b200.solver import MelError
    checkpoints = sorted({k for k in range(5000, args.compare_fp64, 5000)} | {1000, args.compare_fp64})
    rows, done, stopped = [], done0, None
    for k in checkpoints:
        try:
            a.step(k - done)
            b.step(k - done)
            c.step(k - done)
        except MelError as e:          # the sample diverged (both forms run the same physics)
            stopped = {"after_steps": done, "error": str(e)}
            break
        done = k
        ma, mb, mc = a.monitor(), b.monitor(), c.monitor()

        def errs(m):
            return {"kinetic_energy": rel(m.kinetic_energy, ma.kinetic_energy),
                    "wall_contact_force": rel(list(m.rigid_force), list(ma.rigid_force)),
                    "wall_reaction": rel(list(m.rigid_dirichlet), list(ma.rigid_dirichlet)),
                    "mean_displacement": rel(list(m.mean_displacement), list(ma.mean_displacement))}
        row = {"steps": k}
        row.update(errs(mb))
        row["active_contacts"] = [mb.active_contacts, ma.active_contacts]
        row["fp64_twin"] = errs(mc)
        rows.append(row)
    print(json.dumps({"report": "mixed vs fp64 (relative errors; active_contacts = [mixed, fp64]); fp64_twin: "
                                "an FP64 run whose displacement parameters moved by 1e-16 m at step 100, against the FP64 run",
                      "workload": f"biaxial {args.discs} discs", "rows": rows, "diverged": stopped}), flush=True)
    a.close()
    b.close()
    c.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=DEFAULT_STEPS)
    ap.add_argument("--warmup", type=int, default=DEFAULT_WARMUP)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--discs", type=int, default=2000)
    ap.add_argument("--e2e-steps", type=int, default=500)
    # reference sample: enough bodies that its OpenMP loops over bodies keep every host thread busy
    ap.add_argument("--ref-discs", type=int, default=400)
    ap.add_argument("--ref-steps", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # fp64: the drop-in path, bit-identical to the oracle; mixed: FP32 shape-function derivatives,
    # strain and stress with FP64 positions, velocities, contact geometry and force sums
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--compare-fp64", type=int, default=0, metavar="K",
                    help="instead of timing, report the mixed form's errors against FP64 after K steps")
    ap.add_argument("--mode", default="single", choices=["single", "batch", "serve"],
                    help="single: the 2000-disc sample; batch: many independent samples in one batch; "
                         "serve: a Poisson request stream served by continuous batching")
    ap.add_argument("--rate", type=float, default=2.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--drain", type=float, default=60.0)
    ap.add_argument("--step-cap", type=int, default=40000)
    ap.add_argument("--hbm-budget", type=float, default=150.0, help="GB")
    ap.add_argument("--samples", type=int, default=256)
    ap.add_argument("--sample-steps", type=int, default=20000)
    ap.add_argument("--plain-subset", type=int, default=8)
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--accuracy-samples", type=int, default=4)
    # the reference arm: steps of the reference's own loop timed on the full sample
    ap.add_argument("--ref-arm-steps", type=int, default=1000)
    # headline blocks of the default line (one GPU): batched slice and short serving run
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--batch-samples", type=int, default=32)
    ap.add_argument("--batch-plain-subset", type=int, default=4)
    ap.add_argument("--batch-accuracy-samples", type=int, default=2)
    ap.add_argument("--batch-accuracy-steps", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=2.0)
    ap.add_argument("--serve-duration", type=float, default=8.0)
    ap.add_argument("--serve-drain", type=float, default=60.0)
    ap.add_argument("--serve-step-cap", type=int, default=2000)
    ap.add_argument("--mls-discs", type=int, default=400)
    ap.add_argument("--mls-cpu-bodies", type=int, default=20)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_setup()
    try:
        if args.compare_fp64 > 0:
            compare_precisions(args, rank, world, local, pg)
        elif args.mode == "batch" and args.impl == "ours":
            run_batch(args, rank, world, local, pg)
        elif args.mode == "serve" and args.impl == "ours":
            run_serve(args, rank, world, local, pg)
        elif args.impl == "reference":
            run_reference(args, rank, world, pg)
        else:
            run_ours(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
