"""bench.py's multi-rank arithmetic on two CPU ranks (gloo): the device time
of a run is the maximum over ranks, and the whole-job rate counts every
rank's box (weak scaling, one box per GPU, no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, ms_per_rank, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.reduce_max(ms_per_rank[rank], world, "cpu")
        # a second collective in the same order on every rank (the e2e leg)
        ms2 = bench.reduce_max(10.0 * ms_per_rank[rank], world, "cpu")
        out.put((rank, ms, ms2, bench.whole_job_rate(1000, 20, world, ms)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_max_over_ranks_and_whole_job_rate():
    world, port = 2, _free_port()
    ms_per_rank = [3.0, 5.0]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, ms_per_rank, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(out.get(timeout=10) for _ in range(world))
    for rank, ms, ms2, rate in res:
        assert ms == 5.0 and ms2 == 50.0
        # 2 ranks x 1000 cells x 20 steps in 5 ms = 8 MLUPS
        assert rate == pytest.approx(8.0)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(4.25, 1, "cpu") == 4.25
    assert bench.whole_job_rate(1000, 20, 1, 5.0) == pytest.approx(4.0)
