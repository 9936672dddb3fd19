"""GPU primal-dual solvers vs the FP64 oracle.

* per-iteration parity: the GPU iterate after k iterations (no stopping, no
  reweighting) within 2e-5 relative of the oracle's for k <= 20;
* final reconstruction: same stopping rule and reweighting on both, final
  SNR (against the ground-truth cube) within 0.05 dB of the oracle's.
"""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import rel
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry

pytestmark = pytest.mark.gpu

ITER_TOL = 2e-5
SNR_TOL_DB = 0.05


def _setup(algo, Ny=64, Nx=64, L=4, seed=3, Q=(2, 2), overlap=(6, 6), splits=((0, 30, 64), (0, 36, 64))):
    from fhs_b200 import MeasurementOperator
    M = Ny * Nx // 2 if L > 1 else 2 * Ny * Nx
    data, x, meta = problem.make_problem(Ny, Nx, L, M, 2 if L > 1 else 1, seed=seed, synth=synth)
    nu2 = so.operator_norm(data, 200, 1e-10)
    if algo == "fhs":
        geom = FacetGeometry(Ny, Nx, Q[0], Q[1], overlap, splits_y=splits[0], splits_x=splits[1])
    else:
        geom = FacetGeometry(Ny, Nx, 1, 1, (0, 0), window_type="none")
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs" if algo == "fhs" else "hs",
                                              geom if algo == "fhs" else None, nu2)
    if algo == "sara":
        sig = np.sqrt(1.0 / nu2[0])
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    return data, x, op, geom, nu2, sig, sig_bar


def _params(nu2, sig, sig_bar, **kw):
    p = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar)
    p.update(kw)
    return p


def _gpu_solver(algo, op, param, geom, data):
    from fhs_b200 import Solver
    from fhs_b200._lib import ALGO_FHS, ALGO_HS, ALGO_SARA
    a = {"fhs": ALGO_FHS, "hs": ALGO_HS, "sara": ALGO_SARA}[algo]
    kw = {}
    if algo == "fhs":
        kw = dict(Qy=geom.Qy, Qx=geom.Qx, overlap=(geom.base_y[1][0] - geom.over_y[1][0],
                                                   geom.base_x[1][0] - geom.over_x[1][0]),
                  splits_y=[r[0] for r in geom.base_y] + [geom.Ny],
                  splits_x=[r[0] for r in geom.base_x] + [geom.Nx])
    s = Solver(op, a, param, **kw)
    s.set_data(data.y, data.eps)
    s.init()
    return s


def _oracle_run(algo, data, param, geom, max_iter=None):
    p = so.SolverParams(**{k: v for k, v in param.items()})
    if algo == "fhs":
        return so.facet_hypersara(data, p, geom, max_iter=max_iter)
    if algo == "hs":
        return so.hypersara(data, p, max_iter=max_iter)
    xs, log = so.sara(data, p, max_iter=max_iter)
    return xs[None], log


@pytest.mark.parametrize("algo", ["fhs", "hs", "sara"])
def test_iterates_match_oracle(algo):
    L = 1 if algo == "sara" else 4
    data, x, op, geom, nu2, sig, sig_bar = _setup(algo, L=L)
    param = _params(nu2, sig, sig_bar, pdfb_min_iter=10 ** 6, reweighting_flag=False)
    s = _gpu_solver(algo, op, param, geom, data)
    done = 0
    for k in (1, 5, 20):
        s.iterate(k - done)
        done = k
        xo, _ = _oracle_run(algo, data, param, geom, max_iter=k)
        assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL, f"{algo} iteration {k}"
    s.close()


@pytest.mark.parametrize("algo", ["fhs", "hs", "sara"])
def test_final_snr_matches_oracle(algo):
    L = 1 if algo == "sara" else 4
    data, x, op, geom, nu2, sig, sig_bar = _setup(algo, L=L, seed=5)
    param = _params(nu2, sig, sig_bar, pdfb_min_iter=10, pdfb_max_iter=120, reweighting_max_iter=1)
    s = _gpu_solver(algo, op, param, geom, data)
    info = s.run()
    xg = np.moveaxis(s.x(), 2, 0)
    s.close()
    xo, log = _oracle_run(algo, data, param, geom)
    snr_g, snr_o = so.snr_db(x, xg), so.snr_db(x, xo)
    assert abs(snr_g - snr_o) < SNR_TOL_DB, (snr_g, snr_o, info, log.n_iter)
    assert snr_o > 15.0


def test_fhs_iterations_match_golden_fixture():
    """Three GPU FHS iterations against the committed FP64 fixture."""
    import os

    from fhs_b200 import MeasurementOperator, Solver
    from fhs_b200._lib import ALGO_FHS
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fhs_24x24x2_3iter.npz"))
    om = [(g["om_y0"], g["om_x0"]), (g["om_y1"], g["om_x1"])]
    blocks = [list(b) for b in g["blocks"]]
    op = MeasurementOperator(24, 24, om, blocks, [np.full(len(o[0]), 1.0 / s) for o, s in zip(om, g["sigma"])])
    y = [op.split(0, g["y0"]), op.split(1, g["y1"])]
    eps = [synth.l2_bounds(b) for b in blocks]
    param = dict(nu2=g["nu2"], gamma=float(g["sig"]), gamma0=g["sig_bar"], reweighting_sig=float(g["sig"]),
                 reweighting_sig_bar=g["sig_bar"], pdfb_min_iter=10 ** 6, reweighting_flag=False)
    geom = FacetGeometry(24, 24, 2, 2, (3, 3))
    s = Solver(op, ALGO_FHS, param, Qy=2, Qx=2, overlap=(3, 3),
               splits_y=[r[0] for r in geom.base_y] + [24], splits_x=[r[0] for r in geom.base_x] + [24])
    s.set_data(y, eps)
    s.init()
    s.iterate(3)
    assert rel(np.moveaxis(s.x(), 2, 0), g["x3"]) < ITER_TOL
    s.close()


def test_solver_destroy_after_operator():
    """Destroying the operator before its solver (the order a garbage
    collector may pick) leaves no CUDA error behind for later calls."""
    from fhs_b200 import MeasurementOperator, Solver, proj_l2ball
    from fhs_b200._lib import ALGO_HS
    data, x, op, geom, nu2, sig, sig_bar = _setup("hs", L=2)
    s = Solver(op, ALGO_HS, _params(nu2, sig, sig_bar))
    s.set_data(data.y, data.eps)
    s.init()
    s.iterate(2)
    op.close()
    s.close()
    op2 = MeasurementOperator(op.Ny, op.Nx, [(np.zeros(4), np.zeros(4))])
    v = np.ones(8, dtype=complex)
    assert np.allclose(proj_l2ball(v, 1.0, 0 * v), v / np.sqrt(8))
    op2.close()


@pytest.mark.parametrize("algo", ["fhs", "hs"])
def test_noise_adjustment_run_matches_oracle(algo):
    """fhs_solver_run with adjust_flag_noise against the oracle loop: same
    adjustment iterations, adapted l2 bounds and regularisation parameters,
    iterates 5e-5 relative after 26 iterations (two adjustments on the way)."""
    L = 4
    data, x, op, geom, nu2, sig, sig_bar = _setup(algo, Ny=48, Nx=48, L=L, seed=5, Q=(2, 2), overlap=(5, 5),
                                                  splits=((0, 22, 48), (0, 25, 48)))
    data.eps = [[0.3 * e for e in el] for el in data.eps]
    param = _params(nu2, sig, sig_bar, pdfb_min_iter=10 ** 6, pdfb_max_iter=8, reweighting_flag=False,
                    adjust_flag_noise=True, adjust_noise_min_iter=5, adjust_noise_start_iter=3)
    s = _gpu_solver(algo, op, param, geom, data)
    info = s.run(26)
    xo, log = _oracle_run(algo, data, param, geom, max_iter=26)
    assert info["n_iter"] == 26 and info["n_noise_adjustments"] == log.n_adjust >= 2
    assert rel(np.moveaxis(s.x(), 2, 0), xo) < 5e-5
    for eg, eo in zip(s.epsilon(), log.epsilon_final):
        assert np.allclose(eg, eo, rtol=1e-5)
    s.close()


def test_partitioned_driver_matches_solver_run():
    """fhs_b200.distributed.run_partitioned over the library solver (two
    spectral sub-cubes on this GPU, world size 1) takes the same stopping and
    reweighting decisions as fhs_solver_run and ends on the same cube."""
    from fhs_b200 import Solver
    from fhs_b200 import distributed as fd
    from fhs_b200._lib import ALGO_FHS
    data, x, op, geom, nu2, sig, sig_bar = _setup("fhs", L=4, seed=9)
    param = _params(nu2, [sig, sig], np.tile(sig_bar, 2), pdfb_min_iter=4, pdfb_max_iter=12,
                    reweighting_max_iter=2)
    kw = dict(n_groups=2, Qy=2, Qx=2, overlap=(6, 6), splits_y=[0, 30, 64], splits_x=[0, 36, 64])
    s1 = Solver(op, ALGO_FHS, param, **kw)
    s1.set_data(data.y, data.eps)
    s1.init()
    info1 = s1.run()
    s2 = Solver(op, ALGO_FHS, param, **kw)
    s2.set_data(data.y, data.eps)
    s2.init()
    info2 = fd.run_partitioned(fd.GpuSubcubes(s2, 2, 2), 2, [0, 1], param)
    assert (info2["n_iter"], info2["n_reweights"]) == (info1["n_iter"], info1["n_reweights"])
    assert rel(s2.x(), s1.x()) < 1e-7
    s1.close()
    s2.close()
