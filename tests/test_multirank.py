"""The N > 1 path of bench.py on CPU: gloo process groups of two ranks (the GPU
path launches the same way under torchrun with NCCL).  Every rank advances its
own cavity (replicas, no data-path collective); the job's time is the slowest
rank's and its rate counts every rank's work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        secs = [0.5, 2.0][rank]                       # rank 1 is the slow one
        t = bench.max_over_ranks(secs, device="cpu")
        out[rank] = (t, bench.job_rate(1e9, t, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of this threaded process
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 1.0)             # 2 ranks x 1e9 DOF-stages / 2 s


def test_max_over_ranks_without_a_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")),
                    reason="oracle not built")
def test_reference_arm_under_torchrun_prints_one_line():
    """bench.py --impl reference with two ranks: rank 0 times the reference's CPU
    path and prints the one JSON line; rank 1 exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
