"""Visibility gridding (dimensionality reduction) on the GPU vs the FP64
oracle (oracle/dr.py, util_load_data_gen_dr_measurement_operator.m:109-228).

Tolerances: the active set W is exact; diag(H) = Lambda^-2 1e-6 of its
largest entry (FP32 tap polynomials, FP64 sums); operators, reduced data, l2 bounds, dual step 1e-5 relative
(FP32 stencil of FP64 sums, FP32 FFTs); operator norms 1e-4; solver iterates
2e-5 relative, as the visibility solvers.
"""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import rel
from oracle import dr as odr
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
ITER_TOL = 2e-5


def _problem(Ny=32, Nx=40, L=2, M=1500, nb=2, seed=4):
    from fhs_b200 import MeasurementOperator
    data, x, meta = problem.make_problem(Ny, Nx, L, M, nb, seed=seed, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    rng = np.random.default_rng(seed + 100)
    noise = [[(rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b))) / np.sqrt(2) for b in yl]
             for yl in data.y]
    ddr, ops = odr.dr_data_term(data, noise=noise)
    dr = op.dimensionality_reduction()
    return data, x, op, dr, ddr, ops, noise


def _top_eig(data):
    """Largest eigenvalue of Re(A^H Gdr^H Gdr A) per channel (Lanczos, FP64)."""
    from scipy.sparse.linalg import LinearOperator, eigsh
    op = data.op
    out = []
    for l in range(data.L):
        Gd = data.G[l][0]

        def mv(v, Gd=Gd):
            Fx = op.A(np.asarray(v).reshape(op.Ny, op.Nx))
            return np.real(op.At(Gd.conj().T @ (Gd @ Fx))).ravel()
        Lop = LinearOperator((op.Ny * op.Nx,) * 2, matvec=mv, dtype=np.float64)
        out.append(eigsh(Lop, k=1, which="LA", tol=1e-12)[0][0])
    return np.array(out)


def _check_lambda(got, ref):
    """diag(H) = Lambda^-2 to 1e-6 of its largest entry: the FP32 tap
    polynomials carry ~1e-7 absolute error, so cells reached only by the
    small edge taps of a few visibilities have larger relative errors."""
    d_got, d_ref = got ** -2.0, ref ** -2.0
    assert np.abs(d_got - d_ref).max() <= 1e-6 * d_ref.max()
    assert np.median(np.abs(got / ref - 1)) < 1e-6


def test_dr_build_matches_oracle():
    data, x, op, dr, ddr, ops, noise = _problem()
    assert dr.is_dr and not op.is_dr
    for l, (H, W, lam) in enumerate(ops):
        assert np.array_equal(dr.W[l], np.flatnonzero(W))
        assert dr.n_vis[l] == W.sum() and dr.block_sizes[l] == [W.sum()]
        _check_lambda(dr.Lambda[l], lam)
    # gridded data and gridded-noise l2 bounds
    yd = op.reduce_data(dr, data.y)
    nd = op.reduce_data(dr, noise)
    for l in range(data.L):
        assert rel(yd[l][0], ddr.y[l][0]) < OP_TOL
        assert abs(np.linalg.norm(nd[l][0]) - ddr.eps[l][0]) < OP_TOL * ddr.eps[l][0]


def test_dr_operators_match_oracle_and_are_adjoint():
    from fhs_b200 import (HS_adjoint_operator_G, HS_forward_operator_G, apply_adjoint_operator,
                          apply_direct_operator)
    data, x, op, dr, ddr, ops, _ = _problem(L=3, seed=6)
    yg = HS_forward_operator_G(np.moveaxis(x, 0, 2), dr)
    for l, (H, W, lam) in enumerate(ops):
        yo = odr.dr_forward(H, lam, data.op.A(x[l])[W])   # the reference's istril formula
        assert rel(yg[l][0], yo) < OP_TOL
    rng = np.random.default_rng(1)
    v = [[rng.standard_normal(n) + 1j * rng.standard_normal(n)] for n in dr.n_vis]
    xg = np.moveaxis(HS_adjoint_operator_G(v, dr), 2, 0)
    for l, (H, W, lam) in enumerate(ops):
        g2 = np.zeros(data.op.No, dtype=complex)
        g2[W] = odr.dr_adjoint(H, lam, v[l][0])
        assert rel(xg[l], np.real(data.op.At(g2))) < OP_TOL
    lhs = sum(np.vdot(yg[l][0], v[l][0]).real for l in range(data.L))
    rhs = float(np.sum(x * xg))
    assert abs(lhs - rhs) < 1e-5 * abs(rhs)
    # per-channel apply_direct / apply_adjoint on a grid vector
    Fx = rng.standard_normal(dr.No) + 1j * rng.standard_normal(dr.No)
    H, W, lam = ops[1]
    assert rel(apply_direct_operator(Fx, dr, 1), odr.dr_forward(H, lam, Fx[W])) < OP_TOL
    g = apply_adjoint_operator(v[1][0], dr, 1)
    assert rel(g[W], odr.dr_adjoint(H, lam, v[1][0])) < OP_TOL
    assert np.all(g[~W] == 0)


def test_dr_dual_step_norm_and_residuals():
    from fhs_b200 import compute_residual_images, update_dual_data_fidelity
    data, x, op, dr, ddr, ops, _ = _problem(L=2, seed=8)
    rng = np.random.default_rng(3)
    v2 = [[np.linalg.norm(yl[0]) / np.sqrt(len(yl[0])) * (rng.standard_normal(len(yl[0])) +
                                                          1j * rng.standard_normal(len(yl[0])))]
          for yl in ddr.y]
    Fx_old = np.stack([data.op.A(0.8 * x[l]) for l in range(2)])
    s22 = np.array([0.5, 0.25])
    ref = so.update_dual_data_fidelity(v2, 0.9 * x, Fx_old, ddr, s22)
    v2g, Ftx, Fx_new, norm_res, gres, geps = update_dual_data_fidelity(
        v2, ddr.y, np.moveaxis(0.9 * x, 0, 2), Fx_old.T, dr, ddr.eps, s22)
    for l in range(2):
        assert rel(v2g[l][0], ref[0][l][0]) < OP_TOL
        assert np.allclose(norm_res[l], ref[3][l], rtol=1e-5)
    assert rel(np.moveaxis(Ftx, 2, 0), ref[1]) < OP_TOL
    assert abs(gres - ref[4]) < 1e-5 * ref[4] and abs(geps - ref[5]) < 1e-12 * ref[5]
    nu = dr.operator_norm(3000, 1e-12)
    assert np.allclose(nu, _top_eig(ddr), rtol=1e-4), (nu, _top_eig(ddr))
    res = compute_residual_images(np.moveaxis(0.9 * x, 0, 2), ddr.y, dr)
    assert rel(np.moveaxis(res, 2, 0), so.compute_residual_images(0.9 * x, ddr)) < 1e-4


@pytest.mark.parametrize("algo", ["fhs", "sara"])
def test_dr_solver_iterates_match_oracle(algo):
    from fhs_b200 import Solver
    from fhs_b200._lib import ALGO_FHS, ALGO_SARA
    Ny = Nx = 48
    L = 1 if algo == "sara" else 4
    data, x, op, dr, ddr, ops, _ = _problem(Ny, Nx, L, 2 * Ny * Nx // L, 2, seed=12)
    nu2 = so.operator_norm(ddr, 200, 1e-10)
    if algo == "fhs":
        geom = FacetGeometry(Ny, Nx, 2, 2, (5, 5))
        sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
        kw = dict(Qy=2, Qx=2, overlap=(5, 5), splits_y=[r[0] for r in geom.base_y] + [Ny],
                  splits_x=[r[0] for r in geom.base_x] + [Nx])
    else:
        geom = FacetGeometry(Ny, Nx, 1, 1, (0, 0), window_type="none")
        sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "hs", None, nu2)
        sig = np.sqrt(1.0 / nu2[0])
        kw = {}
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    s = Solver(dr, ALGO_FHS if algo == "fhs" else ALGO_SARA, param, **kw)
    s.set_data(ddr.y, ddr.eps)
    s.init()
    p = so.SolverParams(**param)
    done = 0
    for k in (1, 5, 20):
        s.iterate(k - done)
        done = k
        if algo == "fhs":
            xo, _ = so.facet_hypersara(ddr, p, geom, max_iter=k)
        else:
            xs, _ = so.sara(ddr, p, max_iter=k)
            xo = xs[None]
        assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL, f"{algo} iteration {k}"
    s.close()


def test_dr_dense_tile_and_empty_channel():
    """6000 visibilities on a 16 x 16 grid (every cell of a build block reached
    by hundreds of visibilities; the apply tile wraps around the grid) and a
    channel without visibilities (empty W)."""
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G, MeasurementOperator
    from helpers import coverage
    from oracle.nufft import NufftOperator
    Ny = Nx = 8
    oy, ox = coverage(6000, 21)
    om = [(oy, ox), (np.zeros(0), np.zeros(0))]
    op = MeasurementOperator(Ny, Nx, om, [[3000, 3000], [0]])
    ref = NufftOperator(Ny, Nx)
    G = ref.G(oy, ox)
    dr = op.dimensionality_reduction()
    H, W, lam = odr.dr_operator([G[:3000], G[3000:]], ref.No)
    assert np.array_equal(dr.W[0], np.flatnonzero(W)) and dr.n_vis[1] == 0
    _check_lambda(dr.Lambda[0], lam)
    xim = synth.sky_cube(Ny, Nx, 2, 3)
    yg = HS_forward_operator_G(np.moveaxis(xim, 0, 2), dr)
    assert rel(yg[0][0], odr.dr_forward(H, lam, ref.A(xim[0])[W])) < OP_TOL
    assert len(yg[1][0]) == 0
    v = [[np.random.default_rng(0).standard_normal(dr.n_vis[0]) + 0j], [np.zeros(0, complex)]]
    xa = np.moveaxis(HS_adjoint_operator_G(v, dr), 2, 0)
    g2 = np.zeros(ref.No, dtype=complex)
    g2[W] = odr.dr_adjoint(H, lam, v[0][0])
    assert rel(xa[0], np.real(ref.At(g2))) < OP_TOL
    assert np.all(xa[1] == 0)
