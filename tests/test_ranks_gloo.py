"""The multi-rank plumbing of bench.py on CPU: world size 2 over gloo.

Ranks are job replicas with no collective in their data path; the only
exchange is the max over ranks of each timed region.  Checked here without a
GPU: the reduction, the whole-job throughput and the per-rank seeds.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        assert bench.dist_env() == (rank, rank, world)
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, device="cpu")
        out.put((rank, ms, bench.whole_job_rate(3 * 5, world, ms), bench.rank_seed(2, rank)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slower rank's 15 ms; 2 x 15 jobs in 15 ms
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2] == pytest.approx(2 * 15 / 0.015)
    # replicas draw distinct catalogues
    assert res[0][3] != res[1][3]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, device="cpu") == 12.5
    assert bench.whole_job_rate(15, 1, 15.0) == pytest.approx(1000.0)
