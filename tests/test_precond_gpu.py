"""Preconditioned data term on the GPU vs the FP64 oracle: the uniform-weight
preconditioner, the preconditioned operators and norm, the ellipsoid-projection
dual step (src/update_dual_data_fidelity.m:126-147) and the solvers with it.

Tolerances: the preconditioner is integer counting (exact); operators 1e-5
relative (FP32 NUFFT); the dual step 1e-5 relative; solver iterates 2e-5
relative after 1, 5 and 20 iterations, as the pU = 1 solvers.
"""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import coverage, rel
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
ITER_TOL = 2e-5


def _precond(meta, Ky, Kx):
    out = []
    for (oy, ox), sizes in zip(meta["om"], meta["blocks"]):
        pu = so.uniform_weight_preconditioner(oy, ox, Ky, Kx)
        blocks, pos = [], 0
        for m in sizes:
            blocks.append(pu[pos:pos + m])
            pos += m
        out.append(blocks)
    return out


def _problem(Ny=48, Nx=40, L=3, M=2500, nb=2, seed=9):
    from fhs_b200 import MeasurementOperator
    data, x, meta = problem.make_problem(Ny, Nx, L, M, nb, seed=seed, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    pU = _precond(meta, op.Ky, op.Kx)
    op.set_preconditioner(pU)
    return data, x, meta, op, pU


def test_gen_preconditioning_matrix_matches_oracle():
    from fhs_b200 import gen_preconditioning_matrix
    om_y, om_x = coverage(20000, 3)
    for K, sub in ((96, 1), (64, 2)):
        got = gen_preconditioning_matrix(om_y, om_x, K, K, sub)
        ref = so.uniform_weight_preconditioner(om_y, om_x, K * sub, K * sub)
        assert np.array_equal(got, ref)


def test_precond_operators_match_oracle_and_are_adjoint():
    from fhs_b200 import HS_adjoint_operator_precond_G, HS_forward_operator_precond_G
    data, x, meta, op, pU = _problem()
    yg = HS_forward_operator_precond_G(np.moveaxis(x, 0, 2), op)
    yo = so.forward_operator(x, data, pU)
    for l in range(data.L):
        assert rel(np.concatenate(yg[l]), np.concatenate(yo[l])) < OP_TOL
    rng = np.random.default_rng(2)
    v = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in data.y]
    xg = HS_adjoint_operator_precond_G(v, op)
    xo = so.adjoint_operator(v, data, pU)
    assert rel(np.moveaxis(xg, 2, 0), xo) < OP_TOL
    # <Phi x, v> = <x, Phi^H v> (real part: the adjoint keeps real(At(.)))
    lhs = sum(np.vdot(np.concatenate(yg[l]), np.concatenate(v[l])).real for l in range(data.L))
    rhs = float(np.sum(np.moveaxis(x, 0, 2) * xg))
    assert abs(lhs - rhs) < 1e-5 * abs(rhs)


def test_precond_operator_norm_matches_oracle():
    """The top two eigenvalues of Phi^H Phi lie within 0.3% here, so the power
    iteration needs thousands of steps; the reference value is the dense
    eigenvalue of the oracle's operator."""
    data, x, meta, op, pU = _problem(L=1)
    got = op.operator_norm(4000, 1e-12, precond=True)
    N = op.Ny * op.Nx
    cols = []
    for j in range(N):
        e = np.zeros(N)
        e[j] = 1.0
        Fx = data.op.A(e.reshape(op.Ny, op.Nx))
        cols.append(np.concatenate([np.sqrt(p) * (G @ Fx) for G, p in zip(data.G[0], pU[0])]))
    Phi = np.array(cols).T
    ref = np.linalg.eigvalsh((Phi.conj().T @ Phi).real)[-1]
    assert abs(got[0] - ref) < 1e-4 * ref, (got, ref)
    plain = op.operator_norm(4000, 1e-12)
    assert got[0] < plain[0]  # pU <= 1 shrinks the norm


@pytest.mark.parametrize("v2_scale", [10.0, 0.0])
def test_update_dual_data_fidelity_precond_one_step(v2_scale):
    from fhs_b200 import update_dual_data_fidelity_precond
    data, x, meta, op, pU = _problem(L=3, nb=3)
    rng = np.random.default_rng(1)
    v2 = [[v2_scale * (rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b))) for b in yl]
          for yl in data.y]
    proj = [[0.3 * yb for yb in yl] for yl in data.y]
    xk = x * 0.9
    Fx_old = np.stack([data.op.A(x[l] * 0.8) for l in range(3)])
    sigma22 = np.array([0.3, 0.2, 0.1])
    ref = so.update_dual_data_fidelity_precond(v2, proj, xk, Fx_old, data, pU, sigma22, 20, 1, 1e-8)
    v2g, Ftx, Fx_new, pjg, norm_res, gres, geps, its = update_dual_data_fidelity_precond(
        v2, data.y, np.moveaxis(xk, 0, 2), Fx_old.T, proj, op, data.eps, 20, 1, 1e-8, sigma22)
    for l in range(3):
        assert rel(np.concatenate(pjg[l]), np.concatenate(ref[1][l])) < OP_TOL
        assert rel(np.concatenate(v2g[l]), np.concatenate(ref[0][l])) < 1e-4
        assert rel(Fx_new[:, l], ref[3][l]) < OP_TOL
        assert np.allclose(norm_res[l], ref[4][l], rtol=1e-5)
        for b in range(3):
            assert 1 <= its[l][b] <= 20
    assert rel(np.moveaxis(Ftx, 2, 0), ref[2]) < 1e-4
    assert abs(gres - ref[5]) / ref[5] < 1e-5 and abs(geps - ref[6]) / ref[6] < 1e-12


def test_ellipse_projection_stops_like_the_oracle():
    """min_itr = max_itr forces exactly that many FB iterations; a loose
    tolerance stops early, after the same count as the oracle's."""
    from fhs_b200 import update_dual_data_fidelity_precond
    data, x, meta, op, pU = _problem(L=2, nb=2, seed=4)
    v2 = [[np.zeros_like(b) for b in yl] for yl in data.y]
    proj = [[np.zeros_like(b) for b in yl] for yl in data.y]
    Fx_old = np.stack([data.op.A(x[l] * 0.5) for l in range(2)])
    s22 = np.ones(2)
    out = update_dual_data_fidelity_precond(v2, data.y, np.moveaxis(x, 0, 2), Fx_old.T, proj, op, data.eps,
                                            7, 7, 1e-8, s22)
    assert all(k == 7 for l in out[7] for k in l)
    out = update_dual_data_fidelity_precond(v2, data.y, np.moveaxis(x, 0, 2), Fx_old.T, proj, op, data.eps,
                                            50, 1, 1e-3, s22)
    counts = []
    for l in range(2):
        Fx = data.op.A(x[l])
        for b, G in enumerate(data.G[l]):
            r2 = G @ (2 * Fx - Fx_old[l])
            _, k = so.proj_ellipse_fb(r2, data.y[l][b], pU[l][b], data.eps[l][b], np.zeros_like(r2), 50, 1, 1e-3)
            counts.append(k)
    got = [k for l in out[7] for k in l]
    assert all(abs(a - b) <= 1 for a, b in zip(got, counts)), (got, counts)


def _solver_setup(algo, seed=3):
    from fhs_b200 import MeasurementOperator
    Ny = Nx = 64
    L = 1 if algo == "sara" else 4
    M = Ny * Nx // 2 if L > 1 else 2 * Ny * Nx
    data, x, meta = problem.make_problem(Ny, Nx, L, M, 2 if L > 1 else 1, seed=seed, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    pU = _precond(meta, op.Ky, op.Kx)
    op.set_preconditioner(pU)
    nu2 = so.operator_norm(data, 200, 1e-10, pU=pU)
    if algo == "fhs":
        geom = FacetGeometry(Ny, Nx, 2, 2, (6, 6))
    else:
        geom = FacetGeometry(Ny, Nx, 1, 1, (0, 0), window_type="none")
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs" if algo == "fhs" else "hs",
                                              geom if algo == "fhs" else None, nu2)
    if algo == "sara":
        sig = np.sqrt(1.0 / nu2[0])
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    return data, x, op, geom, pU, param


@pytest.mark.parametrize("algo", ["fhs", "sara"])
def test_precond_solver_iterates_match_oracle(algo):
    from fhs_b200 import Solver
    from fhs_b200._lib import ALGO_FHS, ALGO_SARA
    data, x, op, geom, pU, param = _solver_setup(algo)
    kw = {}
    if algo == "fhs":
        kw = dict(Qy=2, Qx=2, overlap=(6, 6), splits_y=[r[0] for r in geom.base_y] + [geom.Ny],
                  splits_x=[r[0] for r in geom.base_x] + [geom.Nx])
    s = Solver(op, ALGO_FHS if algo == "fhs" else ALGO_SARA, param, **kw)
    s.set_data(data.y, data.eps)
    s.init()
    p = so.SolverParams(**param)
    pc = so.Precond(pU)
    done = 0
    for k in (1, 5, 20):
        s.iterate(k - done)
        done = k
        if algo == "fhs":
            xo, _ = so.facet_hypersara(data, p, geom, max_iter=k, precond=pc)
        else:
            xs, _ = so.sara(data, p, max_iter=k, precond=pc)
            xo = xs[None]
        assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL, f"{algo} iteration {k}"
    s.close()
