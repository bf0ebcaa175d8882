"""The multi-rank host logic of bench.py, on CPU: two gloo ranks (127.0.0.1) reduce their
timings to the slowest rank's, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (1 + r) ms for the NTT and (10 - r) ms for the MSM
        q.put((rank, bench.max_over_ranks([1.0 + rank, 10.0 - rank])))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == [2.0, 10.0]


def test_max_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]


def _reference_arm(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--ref-msm-log", "8", "--ref-ntt-log", "8"],
                          capture_output=True, text=True, env=env, timeout=300)


def test_reference_arm_runs_on_rank_zero_only():
    other = _reference_arm(1)
    assert other.returncode == 0 and other.stdout.strip() == ""
    first = _reference_arm(0)
    assert first.returncode == 0, first.stderr
    line = json.loads(first.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
