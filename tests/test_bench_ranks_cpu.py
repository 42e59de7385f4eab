"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): each rank
times its own replica, the job time is the maximum over ranks, the value is
the units of all ranks over that time, and the reference arm does its work on
rank 0 only."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [3.0, 5.0][rank]                       # rank 1 is the slow one
        job = bench.max_over_ranks(ms, dist, device="cpu")
        val = bench.aggregate_rate(1000.0, world, job)
        dist.barrier()
        q.put((rank, job, val))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, job, val in res:
        assert job == 5.0
        assert val == pytest.approx(1000.0 * 2 / 5e-3)


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "phase-field-dislocation-dynamics-pfdd-2.x_b200"))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ws = list(range(7))                          # stand-ins for 7 instances
        mine, scaling = bench.shard_instances(ws, rank, world)
        units = 10.0 * len(mine)
        total = bench.sum_over_ranks(units, dist, device="cpu")
        one, sc1 = bench.shard_instances(["grid"], rank, world)
        dist.barrier()
        q.put((rank, mine, scaling, total, one, sc1))
    finally:
        dist.destroy_process_group()


def test_instances_split_over_ranks_gloo():
    """alloy-like workloads: every instance on exactly one rank; the job's
    units are the sum over ranks; a one-grid workload is replicated."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31000 + os.getpid() % 2000
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert sorted(res[0][1] + res[1][1]) == list(range(7))
    assert not set(res[0][1]) & set(res[1][1])
    for rank, mine, scaling, total, one, sc1 in res:
        assert scaling == "strong" and total == 70.0
        assert one == ["grid"] and sc1 == "weak"


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, None) == 7.5
    assert bench.aggregate_rate(10.0, 1, 1000.0) == pytest.approx(10.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    # the 64^3 deck: the default 256x256x128 grid takes minutes of set-up on a few cores
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--workload", "loop64"], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["metric"] and d["unit"] and d["value"] > 0
        assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
        assert d["cpu_baseline"]["kind"] in ("reference", "port")
