"""Multi-GPU is replicas only: each rank renders its own seeded job, with no
data-path collective; the benchmark sums the ranks' voice-samples and takes
the slowest rank's time. The aggregation runs here as two gloo ranks on CPU.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        # rank r rendered (r + 1) * 1e9 voice-samples in (10 + r) ms; e2e 0.5 of that in (20 + r) ms
        out = bench.reduce_over_ranks((rank + 1) * 1e9, (rank + 1) * 0.5e9, 10.0 + rank, 20.0 + rank, "cpu")
        # every rank takes the same collective steps and sees the same result
        dist.barrier()
        q.put((rank, out, bench.dist_env()))
    finally:
        dist.destroy_process_group()


def test_replicas_sum_work_and_take_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (units, e2e_units, ms_t, e2e_s), env in got:
        assert units == 3e9 and e2e_units == 1.5e9
        assert ms_t == 11.0 and e2e_s == 21.0
        assert env[0] == world and env[1] == rank


def test_each_rank_renders_its_own_seeded_job():
    """Rank r runs the workload with seed + r: the replicas' event streams differ."""
    from kestrel_b200 import host as H
    a = H.config_workload("plain", seed=1 + 0)[2]
    b = H.config_workload("plain", seed=1 + 1)[2]
    assert a.seed != b.seed and a.notes == b.notes


def test_served_cpu_baseline_runs_jobs_on_separate_cores():
    """The served configuration's CPU baseline: the job mix through the CPU
    restatement as independent processes (spawned), a bounded sample each."""
    import bench
    r = bench.served_cpu_baseline(2, 1, 0.2, 2, 0.3)
    assert r["kind"] == "port" and r["cores"] == 2 and r["value"] > 0
