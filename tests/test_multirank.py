"""The multi-process path of bench.py on CPU with gloo, world size 2: the host-side reductions
(max over ranks for time, sum over ranks for work) and a torchrun launch of the reference arm,
where rank 0 alone runs and prints and the other rank exits cleanly."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _reduce_worker(rank, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    world, r, local, pg = bench.dist_setup()
    mx = bench.allreduce_max(pg, 1.5 + rank)
    sm = bench.allreduce_sum(pg, 10.0 * (rank + 1))
    bench.barrier(pg)
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as fh:
        json.dump({"world": world, "rank": r, "max": mx, "sum": sm}, fh)
    pg.destroy_process_group()


def test_host_reductions_over_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.start_processes(_reduce_worker, args=(port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for rank in range(2):
        r = json.load(open(tmp_path / f"r{rank}.json"))
        assert r == {"world": 2, "rank": rank, "max": 2.5, "sum": 30.0}


def test_reference_arm_under_torchrun(oracle_built):
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "5", "--warmup", "3",
           "--discs", "4", "--ref-arm-steps", "5"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    r = json.loads(lines[0])
    assert r["impl"] == "reference" and r["n_gpus"] == 2 and r["value"] > 0
    assert r["cpu_baseline"]["kind"] in ("reference", "port") and r["e2e"]["h2d_bytes_per_step"] == 0
