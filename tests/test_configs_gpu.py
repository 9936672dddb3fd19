"""GPU solvers against the FP64 oracle at the sizes of the four workloads the
library is specified on (all seeded and synthetic):

* single-channel SARA, 256 x 256, M = 2N = 131072 visibilities, 40 dB, exactly
  200 primal-dual iterations with one reweighting (pdfb_min_iter =
  pdfb_max_iter = 100, reweighting_max_iter = 1, as src/sara/sara.m:449
  schedules them): iterates after 1, 20 and 200 iterations and the final SNR;
* HyperSARA, 512 x 512 x 20 over 1-2 GHz, M_l = 0.5N, 40 dB, no faceting:
  operator outputs, the adjoint identity, iterates after 1, 5 and 20
  iterations and the final SNR of a 20 + 20 iteration schedule with one
  reweighting (src/hs/hyperSARA.m:565-866);
* Faceted HyperSARA at the precision-study size, reduced to 2 channels:
  2048 x 2048, 4 x 4 facets with 10% overlap, M_l = 0.5N, 30 dB; operators
  and iterates 1-2 (src/fhs/facetHyperSARA.m:701-889);
* one spectral sub-cube of the batched workload: 1024 x 1024 x 16, M_l
  uniform in [0.3N, 1.0N] in 2-6 blocks, 4 x 4 facets with +-15% jitter, 10%
  overlap, triangular window; iterates 1-2.

Tolerances (written here, as specified for the FP32 path against the FP64
oracle): operator outputs 1e-5 relative, adjoint identity 1e-6, iterates
2e-5 relative, final reconstruction SNR 0.05 dB.  The regularisation
parameters come from compute_noise_level with operator norms measured on the
GPU; both sides get the same values.
"""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import rel
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
ADJ_TOL = 1e-6
ITER_TOL = 2e-5
SNR_TOL_DB = 0.05


def _gpu_op(Ny, Nx, meta):
    from fhs_b200 import MeasurementOperator
    return MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                               [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])


def _solver(op, algo, param, geom=None):
    from fhs_b200 import Solver
    from fhs_b200._lib import ALGO_FHS, ALGO_HS, ALGO_SARA
    a = {"fhs": ALGO_FHS, "hs": ALGO_HS, "sara": ALGO_SARA}[algo]
    kw = {}
    if algo == "fhs":
        kw = dict(Qy=geom.Qy, Qx=geom.Qx, overlap=(geom.base_y[1][0] - geom.over_y[1][0],
                                                   geom.base_x[1][0] - geom.over_x[1][0]),
                  splits_y=[r[0] for r in geom.base_y] + [geom.Ny],
                  splits_x=[r[0] for r in geom.base_x] + [geom.Nx])
    return Solver(op, a, param, **kw)


class _Snapshots:
    """Oracle callback keeping copies of the iterate after chosen iterations."""

    def __init__(self, ks):
        self.ks = set(ks)
        self.x = {}

    def __call__(self, t, x):
        if t in self.ks:
            self.x[t] = np.array(x, copy=True)


def _check_operators(op, data, x, tag):
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G
    yo = so.forward_operator(x, data)
    yg = HS_forward_operator_G(np.moveaxis(x, 0, 2), op)
    for l in range(data.L):
        assert rel(np.concatenate(yg[l]), np.concatenate(yo[l])) < OP_TOL, f"{tag}: forward, channel {l}"
    xo = so.adjoint_operator(data.y, data)
    xg = np.moveaxis(HS_adjoint_operator_G(data.y, op), 2, 0)
    assert rel(xg, xo) < OP_TOL, f"{tag}: adjoint"
    # Re<Phi x, y> = <x, Re Phi^H y> on the GPU path (x real)
    lhs = sum(np.vdot(np.concatenate(yv), np.concatenate(ygl)) for yv, ygl in zip(data.y, yg)).real
    rhs = float(np.sum(xg * x))
    assert abs(lhs - rhs) / abs(lhs) < ADJ_TOL, f"{tag}: adjoint identity"


# --------------------------------------------------------------- 256^2 SARA
@pytest.fixture(scope="module")
def sara_256():
    Ny = Nx = 256
    data, x, meta = problem.make_problem(Ny, Nx, 1, 2 * Ny * Nx, 1, seed=2024, synth=synth)
    op = _gpu_op(Ny, Nx, meta)
    nu2 = op.operator_norm(100, 1e-8)
    sig = float(np.sqrt(1.0 / nu2[0]))
    param = dict(nu2=nu2, gamma=sig, gamma0=np.ones(1), reweighting_sig=sig, reweighting_sig_bar=np.ones(1),
                 pdfb_min_iter=100, pdfb_max_iter=100, reweighting_max_iter=1, reweighting_min_iter=1)
    snap = _Snapshots((1, 20))
    xo, log = so.sara(data, so.SolverParams(**param), callback=snap)
    yield dict(data=data, x=x, op=op, param=param, xo=xo[None], log=log, snap=snap)
    op.close()


def test_sara_256_iterates(sara_256):
    d = sara_256
    s = _solver(d["op"], "sara", dict(d["param"], reweighting_flag=False, pdfb_min_iter=10 ** 6))
    s.set_data(d["data"].y, d["data"].eps)
    s.init()
    s.iterate(1)
    assert rel(np.moveaxis(s.x(), 2, 0), d["snap"].x[1]) < ITER_TOL, "iteration 1"
    s.iterate(19)
    assert rel(np.moveaxis(s.x(), 2, 0), d["snap"].x[20]) < ITER_TOL, "iteration 20"
    s.close()


def test_sara_256_final_200_iterations(sara_256):
    d = sara_256
    assert d["log"].n_iter == 200 and d["log"].n_reweights == 1
    s = _solver(d["op"], "sara", d["param"])
    s.set_data(d["data"].y, d["data"].eps)
    s.init()
    info = s.run()
    xg = np.moveaxis(s.x(), 2, 0)
    s.close()
    assert info["n_iter"] == 200 and info["n_reweights"] == 1, info
    assert rel(xg, d["xo"]) < ITER_TOL, "iteration 200"
    snr_g, snr_o = so.snr_db(d["x"], xg), so.snr_db(d["x"], d["xo"])
    assert abs(snr_g - snr_o) < SNR_TOL_DB, (snr_g, snr_o)
    assert snr_o > 15.0


# ------------------------------------------------------- 512^2 x 20 HyperSARA
@pytest.fixture(scope="module")
def hs_512():
    Ny = Nx = 512
    L = 20
    data, x, meta = problem.make_problem(Ny, Nx, L, Ny * Nx // 2, 1, seed=2025, synth=synth)
    op = _gpu_op(Ny, Nx, meta)
    nu2 = op.operator_norm(100, 1e-8)
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "hs", None, nu2)
    sb = np.atleast_1d(sig_bar)
    param = dict(nu2=nu2, gamma=sig, gamma0=sb, reweighting_sig=sig, reweighting_sig_bar=sb,
                 pdfb_min_iter=20, pdfb_max_iter=20, reweighting_max_iter=1, reweighting_min_iter=1)
    snap = _Snapshots((1, 5, 20))
    xo, log = so.hypersara(data, so.SolverParams(**param), callback=snap)
    yield dict(data=data, x=x, op=op, param=param, xo=xo, log=log, snap=snap)
    op.close()


def test_hs_512x20_operators(hs_512):
    d = hs_512
    _check_operators(d["op"], d["data"], d["x"], "512x512x20")


def test_hs_512x20_iterates(hs_512):
    d = hs_512
    s = _solver(d["op"], "hs", dict(d["param"], reweighting_flag=False, pdfb_min_iter=10 ** 6))
    s.set_data(d["data"].y, d["data"].eps)
    s.init()
    done = 0
    for k in (1, 5, 20):
        s.iterate(k - done)
        done = k
        assert rel(np.moveaxis(s.x(), 2, 0), d["snap"].x[k]) < ITER_TOL, f"iteration {k}"
    s.close()


def test_hs_512x20_final_snr(hs_512):
    d = hs_512
    assert d["log"].n_iter == 40 and d["log"].n_reweights == 1
    s = _solver(d["op"], "hs", d["param"])
    s.set_data(d["data"].y, d["data"].eps)
    s.init()
    info = s.run()
    xg = np.moveaxis(s.x(), 2, 0)
    s.close()
    assert info["n_iter"] == 40 and info["n_reweights"] == 1, info
    snr_g, snr_o = so.snr_db(d["x"], xg), so.snr_db(d["x"], d["xo"])
    assert abs(snr_g - snr_o) < SNR_TOL_DB, (snr_g, snr_o)


# --------------------------------- 2048^2 Faceted HyperSARA (2 channels, 30 dB)
def test_fhs_2048_two_channels_operators_and_iterates():
    Ny = Nx = 2048
    L = 2
    data, x, meta = problem.make_problem(Ny, Nx, L, Ny * Nx // 2, 1, seed=2026, snr_db=30.0, synth=synth)
    op = _gpu_op(Ny, Nx, meta)
    _check_operators(op, data, x, "2048x2048x2")
    ov = int(round(0.1 * Ny / 4))
    geom = FacetGeometry(Ny, Nx, 4, 4, (ov, ov))
    nu2 = op.operator_norm(100, 1e-8)
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    snap = _Snapshots((1, 2))
    so.facet_hypersara(data, so.SolverParams(**param), geom, max_iter=2, callback=snap)
    s = _solver(op, "fhs", param, geom)
    s.set_data(data.y, data.eps)
    s.init()
    for k in (1, 2):
        s.iterate(1)
        assert rel(np.moveaxis(s.x(), 2, 0), snap.x[k]) < ITER_TOL, f"iteration {k}"
    s.close()
    op.close()


# ------------------------- one 16-channel sub-cube of the 1024^2 x 64 workload
def test_fhs_1024_subcube_iterates():
    Ny = Nx = 1024
    L = 16
    N = Ny * Nx
    rng = np.random.default_rng(77)
    Ms = [int(m) for m in rng.integers(int(0.3 * N), N + 1, size=L)]
    nbs = [int(b) for b in rng.integers(2, 7, size=L)]
    data, x, meta = problem.make_problem(Ny, Nx, L, Ms, nbs, seed=2027, synth=synth)
    op = _gpu_op(Ny, Nx, meta)
    ov = int(round(0.1 * Ny / 4))
    sy = synth.jittered_splits(4, Ny, 0.15, rng)
    sx = synth.jittered_splits(4, Nx, 0.15, rng)
    geom = FacetGeometry(Ny, Nx, 4, 4, (ov, ov), splits_y=sy, splits_x=sx)
    nu2 = op.operator_norm(100, 1e-8)
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    snap = _Snapshots((1, 2))
    so.facet_hypersara(data, so.SolverParams(**param), geom, max_iter=2, callback=snap)
    del data.G[:]
    s = _solver(op, "fhs", param, geom)
    s.set_data(data.y, data.eps)
    s.init()
    for k in (1, 2):
        s.iterate(1)
        assert rel(np.moveaxis(s.x(), 2, 0), snap.x[k]) < ITER_TOL, f"iteration {k}"
    s.close()
    op.close()
