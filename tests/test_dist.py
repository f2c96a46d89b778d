"""The multi-GPU bench path on CPU: world size 2 over gloo (no GPU).

The job is replicas (every rank renders its own copy of the scene), so the
only cross-rank steps are a barrier and the timing: the whole-job rate is the
units all ranks processed over the slowest rank's time.  The ranks here are
processes started with `spawn`, as torchrun would start them; they exercise
bench.Dist's barrier, max, sum and job_rate over gloo.  A second test runs
`bench.py --impl reference` under torchrun with two processes: rank 0 alone
times the host path and prints the line, the other rank exits without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(1, backend="gloo")
    try:
        d.barrier()
        ms = 10.0 * (rank + 1)                       # rank 1 is the slow one
        units = 1000.0 * (rank + 1)
        out = {"rank": d.rank, "world": d.world, "max": d.max(ms), "sum": d.sum(units),
               "rate": d.job_rate(units, ms)}
    finally:
        d.close()
    q.put(out)


def test_gloo_world_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r["rank"])
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 20.0                      # slowest rank
        assert r["sum"] == 3000.0
        assert r["rate"] == pytest.approx(3000.0 / 0.020)


def test_single_process_dist_is_local():
    sys.path.insert(0, ROOT)
    import bench
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        d = bench.Dist(1)
        assert d.world == 1 and d.pg is None
        assert d.max(3.0) == 3.0 and d.job_rate(100.0, 10.0) == pytest.approx(1e4)
        d.close()
    finally:
        os.environ.update(env)


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--config", "1", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1                            # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["cores"] >= 1 and line["e2e"]["h2d_bytes_per_step"] == 0
