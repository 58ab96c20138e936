"""The multi-rank path on CPU (gloo, world size 2, 127.0.0.1).

bench.py runs one process per GPU; the views shard across ranks as
independent replicas, and the only collectives are the barrier and the max
over ranks of the timed milliseconds.  These tests run that host logic with
two gloo ranks, and the reference arm under torch.distributed.run (rank 0
renders, the other rank exits without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from helpers import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, local_ms, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        value, ms_max = bench.job_views_per_s(local_ms[rank], 64, 5, world)
        out.put((rank, value, ms_max))
    finally:
        dist.destroy_process_group()


def test_job_throughput_is_max_over_ranks_gloo():
    world = 2
    local_ms = [200.0, 250.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, local_ms, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, ms_max in got:
        assert ms_max == 250.0  # every rank sees the slowest rank's time
        assert value == pytest.approx(2 * 64 * 5 / 0.25)


def test_job_throughput_single_rank_has_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert not dist.is_initialized()
    value, ms_max = bench.job_views_per_s(100.0, 64, 5, 1)
    assert ms_max == 100.0 and value == pytest.approx(64 * 5 / 0.1)


def test_reference_arm_under_torchrun_two_ranks():
    """`--impl reference` launched as the driver launches N > 1 runs: one
    JSON line from rank 0, exit 0 on both ranks."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["unit"] == "views/s" and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
