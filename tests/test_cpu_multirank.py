"""The replica path of bench.py with two ranks (gloo, CPU): every rank times its own
block, the job takes the slowest rank's time (all-reduce MAX) and counts every rank's
cells.  No GPU: the per-rank times are planted."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 13.75][rank]           # rank 1 is the slower one
        m = bench.rank_max(ms, dist)
        q.put((rank, m, bench.whole_job_rate(world, 1000, 20, m)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, rate in got:
        assert m == 13.75
        assert rate == pytest.approx(2 * 1000 * 20 / 13.75e-3 / 1e6)


def test_one_rank_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.rank_max(3.0) == 3.0
    assert bench.whole_job_rate(1, 16777216, 20, 12.81) == pytest.approx(16777216 * 20 / 12.81e-3 / 1e6)
