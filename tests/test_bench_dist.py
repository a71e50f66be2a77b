"""bench.py's multi-rank timing on CPU: two gloo ranks, each with its own
time; every rank sees the slowest, and throughput counts both ranks' work
over that time (weak scaling, no collective on the data path)."""
import os
import socket
import sys

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    my_ms = 100.0 + 50.0 * rank                      # rank 1 is the slower one
    slowest = bench.max_over_ranks(dist, my_ms, "cpu")
    out[rank] = (slowest, bench.aggregate(world, 1000, 3, slowest / 1000.0), bench.seed_base(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_report_the_slowest_time_and_the_whole_job_throughput():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 150.0
    # 2 ranks x 1000 paths x 3 steps over 0.15 s
    assert abs(out[0][1] - 2 * 1000 * 3 / 0.15) < 1e-6
    assert out[0][2] != out[1][2]                    # each rank renders its own samples
