"""Seeded wideband imaging problems built through the library itself.

``build_problem`` assembles the batched Faceted HyperSARA workload: a
power-law sky cube, per-channel Gaussian uv coverage scaled by frequency,
visibility counts uniform in [m_lo N, m_hi N] split into random blocks, noise
at a given input SNR (data and G rows whitened), l2 bounds from the chi2
rule, operator norms by power iteration on the GPU, and regularisation
parameters from compute_noise_level (src/heuristics/compute_noise_level.m).
Channels are interleaved over C spectral sub-cubes (channel l belongs to
sub-cube l mod C); inside the library the channels of a sub-cube are
contiguous.
"""
from __future__ import annotations

import numpy as np

from . import heuristics, synth
from ._lib import ALGO_FHS
from .api import HS_forward_operator_G, MeasurementOperator, Solver, gen_preconditioning_matrix


def build_problem(Ny=1024, Nx=1024, L=64, C=4, Q=4, overlap_frac=0.1, jitter=0.15, m_lo=0.3, m_hi=1.0,
                  blocks=(2, 6), snr_db=40.0, seed=0, device=0, opnorm_iter=50, opnorm_tol=1e-6,
                  pdfb_max_iter=2000, reweighting_max_iter=20, precond=False, dr=False):
    """``precond``: attach the uniform-weight preconditioner (the reference's
    default data term) and take nu2 from the preconditioned operator norm.
    ``dr``: visibility gridding (util_load_data_gen_dr_measurement_operator.m):
    the solver runs on the DR operator, with the gridded data and the l2
    bounds of gridded unit-variance (whitened) noise; the visibility operator
    is released once the data are reduced."""
    rng = np.random.default_rng(seed)
    N = Ny * Nx
    lg = L // C
    # internal channel order: sub-cube c holds the channels l = c, c+C, c+2C, ...
    order = [c + C * i for c in range(C) for i in range(lg)]
    nu = synth.frequencies(L)
    x = synth.sky_cube(Ny, Nx, L, seed)                      # [L, Ny, Nx], frequency order
    x_int = np.ascontiguousarray(x[order])
    Ms = rng.integers(int(m_lo * N), int(m_hi * N) + 1, size=L)
    om_y0, om_x0 = synth.base_coverage(int(Ms.max()), seed)
    om, bsz = [], []
    for l in order:
        oy, ox = synth.channel_coverage(om_y0[: Ms[l]], om_x0[: Ms[l]], nu[l], nu[-1])
        om.append((oy, ox))
        bsz.append(synth.split_blocks(int(Ms[l]), int(rng.integers(blocks[0], blocks[1] + 1)), rng))
    # noiseless data through the library, then whitening by the per-channel sigma
    op0 = MeasurementOperator(Ny, Nx, om, bsz, device=device)
    y0 = HS_forward_operator_G(np.moveaxis(x_int, 0, 2), op0)
    op0.close()
    del op0
    sig = []
    y = []
    for i in range(L):
        y0l = np.concatenate(y0[i])
        s = synth.noise_sigma(y0l, snr_db)
        sig.append(s)
        yl = (y0l + s * synth.noise(y0l.size, rng)) / s
        pos, yb = 0, []
        for m in bsz[i]:
            yb.append(yl[pos:pos + m])
            pos += m
        y.append(yb)
    del y0
    op = MeasurementOperator(Ny, Nx, om, bsz, [np.full(len(o[0]), 1.0 / s) for o, s in zip(om, sig)],
                             device=device)
    eps = [synth.l2_bounds(b) for b in bsz]
    n_vis = int(sum(Ms))
    if dr:
        dop = op.dimensionality_reduction()
        y = op.reduce_data(dop, y)
        noise = [synth.noise(int(sum(b)), rng) for b in bsz]
        eps = [[float(np.linalg.norm(v[0]))] for v in op.reduce_data(dop, noise)]
        op.close()
        op = dop
    if precond:
        op.set_preconditioner([gen_preconditioning_matrix(oy, ox, op.Ky, op.Kx) for oy, ox in om])
    nu2 = op.operator_norm(opnorm_iter, opnorm_tol, precond=precond)
    ov = int(round(overlap_frac * min(Ny, Nx) / Q))
    sy = synth.jittered_splits(Q, Ny, jitter, rng)
    sx = synth.jittered_splits(Q, Nx, jitter, rng)
    gam, gam0, rs, rsb = [], [], [], []
    for c in range(C):
        chans = slice(c * lg, (c + 1) * lg)
        s_, sb, *_ = heuristics.compute_noise_level(Ny, Nx, lg, np.ones(lg), "fhs", nu2[chans], sy, sx, (ov, ov))
        gam.append(s_)
        rs.append(s_)
        gam0.extend(sb)
        rsb.extend(sb)
    param = dict(nu2=nu2, gamma=gam, gamma0=gam0, reweighting_sig=rs, reweighting_sig_bar=rsb,
                 pdfb_max_iter=pdfb_max_iter, reweighting_max_iter=reweighting_max_iter)
    return dict(op=op, y=y, eps=eps, x_true=x_int, param=param, splits=(sy, sx), overlap=(ov, ov), C=C, Q=Q,
                order=order, n_vis=n_vis, nu2=nu2, precond=precond, dr=dr)


def make_solver(prob, nlevel=4):
    s = Solver(prob["op"], ALGO_FHS, prob["param"], nlevel, prob["C"], prob["Q"], prob["Q"], prob["overlap"],
               "triangular", prob["splits"][0], prob["splits"][1])
    s.set_data(prob["y"], prob["eps"])
    return s
