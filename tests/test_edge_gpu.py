"""Edge cases of the GPU path against the FP64 oracle.

* dense tiles: more visibilities in one 64x64 tile than one CTA takes, so the
  degridding slices a tile and the gridding sums partial tiles;
* the block limit (16 blocks in a channel), empty blocks and a channel
  without visibilities;
* spectral groups of 32 channels (the fused SARA prox over two staging
  chunks) and of 40 (the unfused analysis + prox path).

Tolerances as in the other parity tests: operators 1e-5, the dual step
1e-5 (v2, Fx) / 1e-4 (Ftx), solver iterates 2e-5 relative.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from fhs_b200 import synth
from helpers import coverage, rel
from oracle import problem
from oracle import solvers as so
from oracle.facets import FacetGeometry
from oracle.nufft import NufftOperator

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
ITER_TOL = 2e-5


def _blocks(v, sizes):
    out, pos = [], 0
    for m in sizes:
        out.append(v[pos:pos + m])
        pos += m
    return out


def _data(Ny, Nx, om, sizes, seed):
    """DataTerm of given coverages and block sizes (weights 1, y = G A x + noise)."""
    ref = NufftOperator(Ny, Nx)
    rng = np.random.default_rng(seed)
    x = synth.sky_cube(Ny, Nx, len(om), seed) if len(om) > 1 else synth.sky_image(Ny, Nx, seed)[None]
    G_all, y_all, eps_all = [], [], []
    for l, ((oy, ox), bs) in enumerate(zip(om, sizes)):
        G = ref.G(oy, ox) if len(oy) else sp.csr_matrix((0, ref.No), dtype=np.complex128)
        yl = G @ ref.A(x[l]) + 0.01 * synth.noise(len(oy), rng)
        G_all.append([G[a:b] for a, b in zip(np.cumsum([0] + bs[:-1]), np.cumsum(bs))])
        y_all.append(_blocks(yl, bs))
        eps_all.append([0.01 * float(np.sqrt(m + 2 * np.sqrt(m))) for m in bs])
    return so.DataTerm(ref, G_all, y_all, eps_all), x


def test_dense_tile_slices_and_block_limit():
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G, MeasurementOperator, \
        update_dual_data_fidelity
    Ny = Nx = 16  # one 64x64 tile of the 2x grid holds every visibility
    om, sizes = [], []
    for l, M in enumerate((20000, 9000)):
        oy, ox = coverage(M, 40 + l)
        om.append((oy, ox))
        sizes.append([M // 16] * 15 + [M - 15 * (M // 16)] if l == 0 else [M])
    data, x = _data(Ny, Nx, om, sizes, 3)
    op = MeasurementOperator(Ny, Nx, om, sizes)
    yg = HS_forward_operator_G(np.moveaxis(x, 0, 2), op)
    yo = so.forward_operator(x, data)
    for l in range(2):
        assert rel(np.concatenate(yg[l]), np.concatenate(yo[l])) < OP_TOL
    rng = np.random.default_rng(1)
    v = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in data.y]
    assert rel(np.moveaxis(HS_adjoint_operator_G(v, op), 2, 0), so.adjoint_operator(v, data)) < OP_TOL
    # dual variables at the data's scale: with |y| >> |v2| the FP32 sum
    # v2 + 2 G x - G x_old - y cancels and the bound no longer measures the kernels
    v2 = [[np.linalg.norm(np.concatenate(yl)) / np.sqrt(sum(map(len, yl))) * b for b in vl]
          for yl, vl in zip(data.y, v)]
    Fx_old = np.stack([data.op.A(x[l] * 0.8) for l in range(2)])
    s22 = np.array([0.5, 0.25])
    ref = so.update_dual_data_fidelity(v2, x * 0.9, Fx_old, data, s22)
    v2g, Ftx, Fx_new, norm_res, gres, geps = update_dual_data_fidelity(
        v2, data.y, np.moveaxis(x * 0.9, 0, 2), Fx_old.T, op, data.eps, s22)
    for l in range(2):
        assert rel(np.concatenate(v2g[l]), np.concatenate(ref[0][l])) < OP_TOL
        assert np.allclose(norm_res[l], ref[3][l], rtol=1e-5)
    assert rel(np.moveaxis(Ftx, 2, 0), ref[1]) < 1e-4


def test_empty_channel_and_empty_blocks():
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G, MeasurementOperator, Solver
    from fhs_b200._lib import ALGO_HS
    Ny = Nx = 32
    oy0, ox0 = coverage(1500, 7)
    oy1, ox1 = coverage(1200, 8)
    om = [(oy0, ox0), (np.zeros(0), np.zeros(0)), (oy1, ox1), (oy0[:700], ox0[:700])]
    sizes = [[0, 1500, 0], [0], [600, 0, 600], [700]]
    data, x = _data(Ny, Nx, om, sizes, 5)
    op = MeasurementOperator(Ny, Nx, om, sizes)
    assert op.n_vis == [1500, 0, 1200, 700]
    yg = HS_forward_operator_G(np.moveaxis(x, 0, 2), op)
    yo = so.forward_operator(x, data)
    for l in (0, 2, 3):
        assert rel(np.concatenate(yg[l]), np.concatenate(yo[l])) < OP_TOL
    assert sum(len(b) for b in yg[1]) == 0
    rng = np.random.default_rng(2)
    v = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in data.y]
    xa = np.moveaxis(HS_adjoint_operator_G(v, op), 2, 0)
    assert rel(xa, so.adjoint_operator(v, data)) < OP_TOL
    assert np.all(xa[1] == 0.0)
    # HyperSARA runs with the empty channel and blocks and matches the oracle
    # (the empty channel's norm is 0: its nu2 is set to 1 as a placeholder)
    sub = so.DataTerm(data.op, [data.G[l] for l in (0, 2, 3)], [data.y[l] for l in (0, 2, 3)],
                      [data.eps[l] for l in (0, 2, 3)])
    nu2 = np.ones(4)
    nu2[[0, 2, 3]] = so.operator_norm(sub, 200, 1e-10)
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, 4, np.ones(4), "hs", None, nu2)
    param = dict(nu2=nu2, gamma=sig, gamma0=np.atleast_1d(sig_bar), reweighting_sig=sig,
                 reweighting_sig_bar=np.atleast_1d(sig_bar), pdfb_min_iter=10 ** 6, reweighting_flag=False)
    s = Solver(op, ALGO_HS, param)
    s.set_data(data.y, data.eps)
    s.init()
    s.iterate(5)
    xo, _ = so.hypersara(data, so.SolverParams(**param), max_iter=5)
    assert np.all(np.isfinite(s.x()))
    assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL
    s.close()


@pytest.mark.parametrize("L", [32, 40])
def test_large_spectral_groups(L):
    """lg = 32: fused SARA prox with two 16-channel staging chunks; lg = 40:
    the unfused analysis + l21 prox path."""
    from fhs_b200 import MeasurementOperator, Solver
    from fhs_b200._lib import ALGO_FHS
    Ny = Nx = 32
    data, x, meta = problem.make_problem(Ny, Nx, L, 400, 1, seed=11, synth=synth)
    op = MeasurementOperator(Ny, Nx, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    nu2 = so.operator_norm(data, 200, 1e-10)
    geom = FacetGeometry(Ny, Nx, 2, 2, (3, 3))
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, L, np.ones(L), "fhs", geom, nu2)
    sig_bar = np.atleast_1d(sig_bar) * np.ones(geom.Q)
    param = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    s = Solver(op, ALGO_FHS, param, Qy=2, Qx=2, overlap=(3, 3),
               splits_y=[r[0] for r in geom.base_y] + [Ny], splits_x=[r[0] for r in geom.base_x] + [Nx])
    s.set_data(data.y, data.eps)
    s.init()
    s.iterate(5)
    xo, _ = so.facet_hypersara(data, so.SolverParams(**param), geom, max_iter=5)
    assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL
    s.close()


def test_single_visibility_blocks():
    """Blocks holding one visibility and a channel with one visibility in all:
    operators and the l2-ball dual step against the oracle.  A single
    visibility's G Fx is a sum of 49 FP32 products that can cancel, so its
    error is measured against the operand scale ||(|G| |Fx|)_b|| (block
    residual norms within 2e-5 of it; the other blocks' observed errors are
    below 2e-6 of it), and v2 is drawn at 10x that scale so that z = v2 +
    2 G Fx - G Fx_old - y does not cancel."""
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G, MeasurementOperator, \
        update_dual_data_fidelity
    Ny, Nx = 32, 24
    oy0, ox0 = coverage(1000, 12)
    om = [(oy0, ox0), (oy0[:1], ox0[:1]), (oy0[:3], ox0[:3])]
    sizes = [[1, 1, 998], [1], [1, 1, 1]]
    data, x = _data(Ny, Nx, om, sizes, 9)
    op = MeasurementOperator(Ny, Nx, om, sizes)
    yg = HS_forward_operator_G(np.moveaxis(x, 0, 2), op)
    yo = so.forward_operator(x, data)
    for l in range(3):
        assert rel(np.concatenate(yg[l]), np.concatenate(yo[l])) < OP_TOL
    rng = np.random.default_rng(4)
    v = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in data.y]
    assert rel(np.moveaxis(HS_adjoint_operator_G(v, op), 2, 0), so.adjoint_operator(v, data)) < OP_TOL
    # FP32 operand scale of G Fx per block, at the dual step's x
    scale = [[float(np.linalg.norm(abs(G) @ abs(data.op.A(0.9 * x[l])))) for G in data.G[l]] for l in range(3)]
    v2 = [[10.0 * np.sqrt(sum(t * t for t in sl) / sum(map(len, yl))) * b for b in vl]
          for yl, vl, sl in zip(data.y, v, scale)]
    Fx_old = np.stack([data.op.A(x[l] * 0.8) for l in range(3)])
    s22 = np.array([0.5, 0.3, 0.2])
    ref = so.update_dual_data_fidelity(v2, x * 0.9, Fx_old, data, s22)
    v2g, Ftx, Fx_new, norm_res, gres, geps = update_dual_data_fidelity(
        v2, data.y, np.moveaxis(x * 0.9, 0, 2), Fx_old.T, op, data.eps, s22)
    for l in range(3):
        assert rel(np.concatenate(v2g[l]), np.concatenate(ref[0][l])) < OP_TOL
        for b in range(len(sizes[l])):
            assert abs(norm_res[l][b] - ref[3][l][b]) <= 2e-5 * scale[l][b], (l, b)
    assert rel(np.moveaxis(Ftx, 2, 0), ref[1]) < 1e-4
