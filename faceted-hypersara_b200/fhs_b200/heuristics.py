"""Regularisation heuristics (host, FP64 scalars).

Restates src/heuristics/compute_noise_level.m:49-89 and
compute_noise_level_sara.m:20: the noise level in the SARA domain (sig) and
in the singular-value domain of every nuclear-norm facet (sig_bar), from the
per-channel noise standard deviations and squared operator norms.
"""
from __future__ import annotations

from math import lgamma

import numpy as np


def split_points(Q: int, N: int) -> list:
    """Facet boundaries of split_range(Q, N): round(linspace(0, N, Q+1))."""
    return [int(np.floor(q * N / Q + 0.5)) for q in range(Q + 1)]


def facet_pixels(splits_y, splits_x, overlap=(0, 0)) -> list:
    """Pixels of every overlapped facet, q = qx*Qy + qy (y fastest)."""
    def sizes(sp, ov):
        out = []
        for q in range(len(sp) - 1):
            a = max(sp[q] - ov, 0) if q > 0 else sp[q]
            out.append(sp[q + 1] - a)
        return out
    sy, sx = sizes(splits_y, overlap[0]), sizes(splits_x, overlap[1])
    return [py * px for px in sx for py in sy]


def compute_noise_level(Ny, Nx, n_channels, std_noise, algo, squared_operator_norm, splits_y=None,
                        splits_x=None, overlap=(0, 0)):
    """Returns (sig, sig_bar, mu_chi, sig_chi, sig_sara); sig_bar per facet for
    'fhs' (facets from splits/overlap), a scalar for 'hs'."""
    std_noise = np.asarray(std_noise, dtype=np.float64).ravel()
    son = np.asarray(squared_operator_norm, dtype=np.float64).ravel()
    L = int(n_channels)
    sig_sara = float(np.sqrt(np.mean(std_noise ** 2 / son)))
    mu_chi = float(np.sqrt(2.0) * np.exp(lgamma((L + 1) / 2.0) - lgamma(L / 2.0)))
    sig_chi = float(np.sqrt(max(L - mu_chi ** 2, 0.0)))
    sig = sig_sara * (mu_chi + sig_chi)
    s = float(np.sum(std_noise ** 2 / son))
    if algo == "hs":
        sig_bar = float(np.sqrt(Nx * Ny * s / min(Nx * Ny, L)))
    else:
        pix = facet_pixels(splits_y, splits_x, overlap)
        sig_bar = np.array([np.sqrt(p * s / min(p, L)) for p in pix])
    return sig, sig_bar, mu_chi, sig_chi, sig_sara


def compute_noise_level_sara(std_noise, squared_operator_norm):
    """src/heuristics/compute_noise_level_sara.m:20."""
    return float(np.sqrt(float(std_noise) ** 2 / float(squared_operator_norm)))


def update_epsilon(epsilon, t, t_block, norm_res, adapt_eps_tol_in, adapt_eps_tol_out, adapt_eps_steps,
                   adapt_eps_change_percentage):
    """src/update_epsilon.m:52-71 (adaptive l2 bounds, the reference's
    use_adapt_eps; its solvers keep the call commented out): for every block
    last changed more than adapt_eps_steps iterations ago, move eps towards
    the residual, eps <- c ||res|| + (1 - c) eps, when ||res|| < tol_in eps
    or ||res|| > tol_out eps.  epsilon, t_block, norm_res: [l][b] lists
    (updated copies returned as (epsilon, t_block))."""
    eps = [list(map(float, e)) for e in epsilon]
    tb = [list(map(int, b)) for b in t_block]
    c = float(adapt_eps_change_percentage)
    for i, (el, rl) in enumerate(zip(eps, norm_res)):
        for j, r in enumerate(rl):
            if t > tb[i][j] + adapt_eps_steps:
                if r < adapt_eps_tol_in * el[j]:
                    el[j] = c * r + (1.0 - c) * el[j]
                    tb[i][j] = t
                if r > adapt_eps_tol_out * el[j]:
                    el[j] = c * r + (1.0 - c) * el[j]
                    tb[i][j] = t
    return eps, tb
