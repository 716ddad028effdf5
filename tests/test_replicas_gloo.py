"""The multi-GPU path of bench.py runs independent replicas (no data-path
collective): each rank times its own RHS evaluations, the job time is the
slowest rank's, and the value is the whole-job rate.  Checked here with two
gloo ranks on the CPU."""
import os
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
        t = bench.max_over_ranks(ms, world, "cpu")
        q.put((rank, t, bench.job_throughput(world, 1000, 4, t)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, v in res:
        assert t == 15.0                        # the slowest rank's time on every rank
        assert abs(v - 2 * 1000 * 4 / 0.015 / 1e6) < 1e-12


def test_reference_arm_idle_on_nonzero_rank():
    class A:
        steps, warmup, gpus = 1, 1, 2
    assert bench.run_reference(A(), rank=1, world=2) == 0
