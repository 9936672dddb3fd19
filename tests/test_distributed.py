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


def test_algorithmic_bytes_per_launch():
    """bench.py's roofline numerators: the per-launch byte formulas of the
    visibility (l2-ball and preconditioned) and DR data terms."""
    from types import SimpleNamespace

    import bench
    L, Ny, Nx, M = 4, 64, 64, 10000
    No = 4 * Ny * Nx
    op = SimpleNamespace(L=L, Ny=Ny, Nx=Nx, No=No, n_vis_total=3000, block_sizes=[[M // L]] * L)
    prob = dict(op=op, n_vis=M, Q=2, splits=([0, 32, 64], [0, 32, 64]), overlap=(4, 4), C=1)
    b = bench.algorithmic_bytes(prob, 9 * Ny * Nx)
    assert b["degrid_dual"] == No * L * 8 + M * 56
    assert b["grid_dual"] == M * 32 + No * L * 8
    bp = bench.algorithmic_bytes(dict(prob, precond=True), 9 * Ny * Nx, [[2] for _ in range(L)])
    assert bp["degrid_dual"] == b["degrid_dual"] + 20 * M and bp["ellipse_fb"] == 2 * M * 53
    bd = bench.algorithmic_bytes(dict(prob, dr=True), 9 * Ny * Nx)
    n = op.n_vis_total
    stencil = n * (85 * 8 + 8) + L * No * 4
    assert bd["degrid_dual"] == stencil + L * (No // 2) * 8 + n * 40
    assert bd["grid_dual"] == stencil + n * 16 + L * No * 8


def test_reference_arm_prints_the_contract_line():
    """bench.py --impl reference (the FP64 oracle on the host cores) prints one
    JSON line with the keys the bench contract asks of the reference arm."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=900, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "iter/s" and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
