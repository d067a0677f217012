"""The N>1 bench path on CPU: two gloo ranks reduce their step timings to the
slowest rank's, and the whole-job rate sums the ranks' work over that time."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        # Rank 0 is slower in the first value, rank 1 in the second.
        times = [10.0 + 5.0 * (rank == 0), 3.0 + 4.0 * (rank == 1), 1.0 + rank]
        got = bench.max_over_ranks(times, dist, "cpu")
        q.put((rank, got, bench.whole_job_rate(world, 1e9, got[0])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [15.0, 7.0, 2.0]
        assert rate == pytest.approx(2 * 1e9 / 0.015)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert bench.whole_job_rate(1, 100.0, 1000.0) == pytest.approx(100.0)
