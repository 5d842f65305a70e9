"""Replica path of bench.py (--gpus N under torchrun) on CPU: two gloo ranks
time different amounts of work; every rank sees the maximum, the whole-job
rate counts both ranks' units over the slowest rank's time, and the
reference arm's non-zero ranks exit without output."""

import os
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from replicas import barrier, max_over_ranks, whole_job_rate
    barrier()
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    m = max_over_ranks(ms)
    rate = whole_job_rate(world, 1000, m)
    barrier()
    out.put((rank, m, rate))
    dist.destroy_process_group()


def test_max_over_ranks_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    assert all(r[2] == pytest.approx(2 * 1000 / 0.020) for r in res)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
