"""Multi-GPU is replicas only: every rank advances its own copy and the bench
takes the slowest rank's time.  The reduction runs here on two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    t = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
    # the aggregate a rank reports: units of all ranks over the slowest time
    value = 1000 * world / t
    q.put((rank, t, value))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert out[0][2] == pytest.approx(800.0)


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25
