"""Multi-rank bench logic on CPU with the gloo backend (world size 2): the
timing is the maximum over ranks on every rank, and the whole-job value
counts every rank's replica (the data path has no collective; ranks only
agree on timings)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r measured (1 + r) ms per step and (10 - r) ms end to end
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
        value = bench.job_value(1e9, got[0], world)
        q.put((rank, got, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, got, value in res:
        assert got == [2.0, 10.0]               # the slowest rank's step, the slowest end to end
        assert value == pytest.approx(1000.0)   # 2 ranks x 1 GFLOP per step / 2 ms


def test_single_process_passthrough():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench.job_value(2e9, 4.0, 1) == pytest.approx(500.0)
