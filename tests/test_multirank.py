"""Host logic of runs on N > 1 GPUs, exercised with world-size-2 gloo process groups on the CPU:
the replicas' job time is the slowest rank's, the whole-job throughput aggregates over ranks,
and the ensemble's arrival stream is dealt to the ranks without overlap or loss."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    from openlb_b200 import serving
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [40.0, 55.0][rank]                   # the second rank is slower
        worst = bench.rank_max(dist, ms)
        reqs = serving.sample_requests(101, seed=9)
        mine = serving.shard_requests(reqs, rank, world)
        ids = [r.rid for r in mine]
        gathered = [None] * world
        dist.all_gather_object(gathered, ids)
        out.put((rank, worst, bench.job_mlups(world, 256 ** 3, 100, worst), gathered))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_aggregate_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for rank, worst, mlups, gathered in results:
        assert worst == 55.0                    # both ranks report the slowest rank's time
        assert mlups == pytest.approx(2 * 256 ** 3 * 100 / 0.055 / 1e6)
        a, b = gathered
        assert not set(a) & set(b) and sorted(a + b) == list(range(101))
        assert abs(len(a) - len(b)) <= 1


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.rank_max(None, 3.5) == 3.5
    assert bench.job_mlups(1, 1000, 10, 1.0) == pytest.approx(10.0)
