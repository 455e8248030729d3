"""Autotuner of the body kernel's chunk size: for each workload class (precision, largest deformable
body) it times the body kernel at every candidate chunk entry cap on a small sample of that class
(CUDA events on the solver's stream, mel_get_kernel_times) and writes the fastest cap to a tuning
table that mel_create reads (environment variable MELGPU_TUNE_FILE; melody2d_b200.solver points it at
melody2d_b200/tuning.txt when that file exists and the variable is unset).

    python -m melody2d_b200.autotune [--out melody2d_b200/tuning.txt] [--discs 300] [--steps 30]

Classes: the 2000-disc workload's discs (64 border + 340 interior nodes) and the largest grains of
the batched workload (96 border + 480 interior nodes), each in FP64 and in mixed precision.  The
chunk cap trades the bytes in flight per SM (larger images) against the number of CTAs that fit an
SM and the per-chunk pipeline overhead; the table lines are "precision max_body_nodes cap"."""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning.txt")
CAPS = [2048, 1792, 1536, 1408, 1280, 1152, 1024, 896, 768]
CAPS_MIXED = [3584, 3328, 3072, 2816, 2560, 2304] + CAPS   # FP32 images: larger chunks fit the same memory
CLASSES = [(64, 340), (96, 480)]          # (border nodes, interior nodes) of the class's discs


def time_cap(flat, precision: int, cap: int, steps: int, warmup: int = 5) -> float:
    """Body-kernel milliseconds per step at chunk cap `cap` (CUDA events)."""
    from melody2d_b200.solver import Solver
    os.environ["MELGPU_CHUNK_CAP"] = str(cap)
    try:
        s = Solver.from_flat(flat, precision=precision)
    finally:
        del os.environ["MELGPU_CHUNK_CAP"]
    try:
        s.step(warmup, proximity=False)
        s.set_timing(True)
        s.step(steps, proximity=False)
        return s.kernel_times()["body"] / steps
    finally:
        s.close()


def tune(out: str, discs: int, steps: int, workers: int) -> dict:
    from melody2d_b200 import generator as g
    rows, report = [], []
    for nb, ni in CLASSES:
        t0 = time.perf_counter()
        flat = g.flatten(g.biaxial_scene(seed=7, n_discs=discs, n_border=nb, n_interior=ni, workers=workers))
        gen_s = time.perf_counter() - t0
        for precision in (0, 1):
            times = {cap: time_cap(flat, precision, cap, steps) for cap in (CAPS_MIXED if precision else CAPS)}
            best = min(times, key=times.get)
            rows.append((precision, nb + ni, best))
            report.append({"precision": ["fp64", "mixed"][precision], "max_body_nodes": nb + ni, "best_cap": best,
                           "body_ms": {str(k): round(v, 5) for k, v in times.items()}, "generate_s": round(gen_s, 1)})
            print(json.dumps(report[-1]), flush=True)
    with open(out, "w") as fh:
        fh.write("# chunk entry cap per (precision 0 fp64 / 1 mixed, largest deformable body in nodes), written by\n"
                 "# python -m melody2d_b200.autotune (body-kernel time on a %d-disc sample of each class)\n" % discs)
        for p, n, c in rows:
            fh.write("%d %d %d\n" % (p, n, c))
    return {"table": out, "classes": report}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--discs", type=int, default=300)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args(argv)
    tune(a.out, a.discs, a.steps, a.workers)
    return 0


if __name__ == "__main__":
    sys.exit(main())
