"""Checkpoint / warm restart through the C ABI: the state read after k
iterations, written to a MAT-file and restored into a fresh solver, continues
exactly like the original solver (same graph, same data: equal to rounding)."""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import rel
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precond", [False, True])
def test_restored_solver_continues_the_run(tmp_path, precond):
    from fhs_b200 import MeasurementOperator, Solver, load_checkpoint, save_checkpoint
    from fhs_b200._lib import ALGO_FHS
    Ny = Nx = 48
    L = 4
    data, x, meta = problem.make_problem(Ny, Nx, L, Ny * Nx // 2, 2, seed=6, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    if precond:
        op.set_preconditioner([so.uniform_weight_preconditioner(oy, ox, op.Ky, op.Kx) for oy, ox in meta["om"]])
    nu2 = op.operator_norm(300, 1e-9, precond=precond)
    geom = FacetGeometry(Ny, Nx, 2, 2, (5, 5))
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    kw = dict(Qy=2, Qx=2, overlap=(5, 5), splits_y=[r[0] for r in geom.base_y] + [Ny],
              splits_x=[r[0] for r in geom.base_x] + [Nx])

    def solver():
        s = Solver(op, ALGO_FHS, param, **kw)
        s.set_data(data.y, data.eps)
        return s

    a = solver()
    a.init()
    a.iterate(6)
    state = a.get_state()
    assert ("proj" in state) == precond
    path = tmp_path / "ckpt.mat"
    save_checkpoint(path, state, end_iter=6)
    a.iterate(4)
    ref = a.x()
    b = solver()
    restored = load_checkpoint(path)
    b.init(restored["xsol"])
    b.set_state(restored)
    b.iterate(4)
    assert rel(b.x(), ref) < 1e-6
    a.close()
    b.close()


def test_restore_after_noise_adjustment(tmp_path):
    """A run whose noise adjustment changed the l2 bounds and the
    regularisation: the checkpoint carries epsilon, and a solver restored from
    it (with the adapted gamma / gamma0) continues the original run."""
    from fhs_b200 import MeasurementOperator, Solver, load_checkpoint, save_checkpoint
    from fhs_b200._lib import ALGO_FHS
    Ny = Nx = 48
    L = 4
    data, x, meta = problem.make_problem(Ny, Nx, L, Ny * Nx // 2, 2, seed=6, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    nu2 = op.operator_norm(300, 1e-9)
    geom = FacetGeometry(Ny, Nx, 2, 2, (5, 5))
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    eps0 = [[0.3 * e for e in el] for el in data.eps]
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, pdfb_max_iter=8, reweighting_flag=False, adjust_flag_noise=True)
    kw = dict(Qy=2, Qx=2, overlap=(5, 5), splits_y=[r[0] for r in geom.base_y] + [Ny],
              splits_x=[r[0] for r in geom.base_x] + [Nx])
    a = Solver(op, ALGO_FHS, param, **kw)
    a.set_data(data.y, eps0)
    a.init()
    info = a.run(6)
    assert info["n_noise_adjustments"] >= 1
    state = a.get_state()
    assert not np.allclose(state["epsilon"][0], eps0[0])
    path = tmp_path / "ckpt.mat"
    save_checkpoint(path, state, end_iter=6)
    g, g0 = a.regularization()
    a.iterate(4)
    ref = a.x()
    b = Solver(op, ALGO_FHS, dict(param, gamma=g, gamma0=g0, adjust_flag_noise=False), **kw)
    b.set_data(data.y, eps0)
    restored = load_checkpoint(path)
    b.init(restored["xsol"])
    b.set_state(restored)
    assert np.allclose(np.concatenate(b.epsilon()), np.concatenate(state["epsilon"]), rtol=0, atol=0)
    b.iterate(4)
    assert rel(b.x(), ref) < 1e-6
    a.close()
    b.close()
