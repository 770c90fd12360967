"""bench.py's multi-rank host logic on CPU: two gloo ranks on 127.0.0.1.

On GPUs the same helpers run over NCCL under torchrun (one replica per GPU,
no data-path collective); here the slowest rank's time must win on every
rank, whole-job ms per mesh must count every rank's meshes, and the
reference arm must print on rank 0 only."""

import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, results):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        slowest = bench.max_over_ranks(10.0 * (rank + 1), 2, torch.device("cpu"))
        results.put((rank, slowest, bench.whole_job_ms_per_mesh(slowest, 5, 2)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(results.get(timeout=10) for _ in range(2))
    assert got == [(0, 20.0, 2.0), (1, 20.0, 2.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.whole_job_ms_per_mesh(30.0, 10, 1) == 3.0


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--config", "icospheres-2560", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == ""
    env["RANK"] = env["LOCAL_RANK"] = "0"
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--config", "icospheres-2560", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
