"""Multi-rank host logic on CPU (gloo, world size 2).

* bench.py: every rank solves its own cube, the timing is the max over ranks
  and the value is the whole-job throughput;
* fhs_b200.distributed: one cube's spectral sub-cubes split over ranks, with
  the stopping statistics all-reduced in FP64 -- the gathered cube equals, bit
  for bit, the run of one process holding every sub-cube (the local work is
  the FP64 oracle's Faceted HyperSARA iteration, as the GPU is not available
  here)."""
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
                        "--warmup", "3", "--case", "small"], capture_output=True, text=True, timeout=900, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "iter/s" and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert "spectral sub-cube" in d["cpu_baseline"]["sample"] and "x4 sub-cubes" in d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


# ------------------------------------------------ sub-cube partition of one cube
_NY = _NX = 32
_L, _C = 4, 2


def _subcube_problem():
    """One 32 x 32 x 4 cube, C = 2 interleaved sub-cubes of 2 channels: per
    sub-cube the oracle data term, facet geometry and parameters."""
    import numpy as np

    from fhs_b200 import synth
    from oracle import problem
    from oracle import solvers as so
    from oracle.facets import FacetGeometry
    data, x, meta = problem.make_problem(_NY, _NX, _L, 400, 2, seed=21, synth=synth)
    nu2 = so.operator_norm(data, 60, 1e-9)
    geom = FacetGeometry(_NY, _NX, 2, 2, (3, 3))
    subs = []
    for c in range(_C):
        ch = list(range(c, _L, _C))
        d = so.DataTerm(data.op, [data.G[l] for l in ch], [data.y[l] for l in ch], [data.eps[l] for l in ch])
        sig, sig_bar, *_ = so.compute_noise_level(_NY, _NX, len(ch), np.ones(len(ch)), "fhs", geom, nu2[ch])
        p = so.SolverParams(nu2=nu2[ch], gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                            pdfb_min_iter=4, pdfb_max_iter=12, reweighting_max_iter=2)
        subs.append((d, p))
    return subs, geom


class _OracleSubcubes:
    def __init__(self, subs, geom, mine):
        from oracle import solvers as so
        self.its = [so.FhsIteration(subs[c][0], subs[c][1], geom) for c in mine]

    def step(self):
        import numpy as np
        return np.array([it.step()[:4] for it in self.its])

    def x(self):
        import numpy as np
        return np.stack([it.x for it in self.its])

    def reweight(self):
        for it in self.its:
            it.reweight()


_PARAM = dict(pdfb_min_iter=4, pdfb_max_iter=12, reweighting_max_iter=2)


def _partition_worker(rank, world, port, q):
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      FHS_ORACLE_THREADS="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for pth in (root, os.path.join(root, "faceted-hypersara_b200"), os.path.join(root, "tests")):
        sys.path.insert(0, pth)
    import torch.distributed as dist

    from fhs_b200 import distributed as fd
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    subs, geom = _subcube_problem()
    mine = fd.subcubes_of_rank(_C, world, rank)
    local = _OracleSubcubes(subs, geom, mine)
    info = fd.run_partitioned(local, _C, mine, _PARAM, dist=dist)
    x = fd.gather_cube(local.x(), _C, _L, mine, world, dist=dist)
    q.put((rank, info, x))
    dist.barrier()
    dist.destroy_process_group()


def test_subcube_partition_matches_one_process():
    import numpy as np

    from fhs_b200 import distributed as fd
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # one process holding both sub-cubes, same driver, no process group
    subs, geom = _subcube_problem()
    local = _OracleSubcubes(subs, geom, [0, 1])
    info1 = fd.run_partitioned(local, _C, [0, 1], _PARAM)
    x1 = fd.gather_cube(local.x(), _C, _L, [0, 1], 1)
    for rank, info, x in out:
        assert info == info1, (rank, info, info1)
        assert np.array_equal(x, x1), rank
    assert info1["n_reweights"] == 2 and info1["n_iter"] > 12
    # the sub-cubes hold the interleaved channels: channel l is sub-cube l mod C
    assert fd.subcubes_of_rank(4, 2, 1) == [1, 3] and fd.channels_of_subcube(1, 4, 16) == [1, 5, 9, 13]
