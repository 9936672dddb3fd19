"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): every rank
solves its own cube, the timing is the max over ranks and the value is the
whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 + 50.0 * rank               # rank 1 is the slow one
    ms_max = bench._max_over_ranks(dist, ms, "cpu")
    q.put((rank, ms_max, bench.aggregate_value(world, 20, ms_max)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_weak_scaling_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [150.0, 150.0]
    assert out[0][2] == pytest.approx(2 * 20 / 0.150)
