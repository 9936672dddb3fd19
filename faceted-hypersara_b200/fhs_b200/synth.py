"""Seeded synthetic wideband radio-interferometric inputs.

Stand-ins for the reference's Cyg A cubes and VLA coverages (not shipped with
the reference).  Shapes and distributions follow the workloads the solver is
measured on:

* sky: nonnegative image of 30 Gaussian blobs (sigma 2-12 px, amplitude
  Exp(1)) plus 200 point sources (amplitude log-uniform in [1e-3, 1]);
* cube: ``x_l(p) = x_ref(p) (nu_l/nu_1)^alpha(p)``, ``alpha ~ N(-0.7, 0.2)``,
  channels linear over 1-2 GHz;
* coverage: ``(u, v) ~ N(0, (pi/4)^2)`` clipped to ``[-pi, pi]`` (the
  reference's ``lib/generate_data/util_gen_sampling_pattern.m:54-87`` rejects
  instead); per channel scaled by ``nu_l / nu_max`` as in
  ``lib/operators/util_gen_measurement_operator_synth.m:70-71``;
* noise: input SNR per channel, ``sigma_l = 10^(-snr/20) ||y0_l|| / sqrt(M_l)``
  (``lib/generate_data/util_gen_measurements_snr_new.m:57``), data and
  operator whitened by ``sigma_l``;
* l2 bounds ``eps_l = sqrt(M_l + 2 sqrt(M_l))`` in the whitened domain, split
  over blocks as ``sqrt(m_b / M_l) eps_l``
  (``lib/utils/util_gen_data_fidelity_bounds2.m:23-36``, ``sigma_ball = 2``).

All helpers are pure NumPy and deterministic in ``seed``.
"""
from __future__ import annotations

import numpy as np


def sky_image(Ny: int, Nx: int, seed: int, n_blobs: int = 30, n_points: int = 200) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = np.zeros((Ny, Nx))
    yy = np.arange(Ny)[:, None]
    xx = np.arange(Nx)[None, :]
    for _ in range(n_blobs):
        cy, cx = rng.uniform(0, Ny), rng.uniform(0, Nx)
        s = rng.uniform(2.0, 12.0)
        a = rng.exponential(1.0)
        gy = np.exp(-0.5 * ((yy - cy) / s) ** 2)
        gx = np.exp(-0.5 * ((xx - cx) / s) ** 2)
        x += a * gy * gx
    py = rng.integers(0, Ny, n_points)
    px = rng.integers(0, Nx, n_points)
    amp = 10.0 ** rng.uniform(-3.0, 0.0, n_points)
    np.add.at(x, (py, px), amp)
    return x


def frequencies(L: int, f0: float = 1e9, f1: float = 2e9) -> np.ndarray:
    return np.linspace(f0, f1, L) if L > 1 else np.array([f0])


def sky_cube(Ny: int, Nx: int, L: int, seed: int, x_ref=None) -> np.ndarray:
    """Power-law cube [L, Ny, Nx] (channel-first)."""
    rng = np.random.default_rng(seed + 7919)
    if x_ref is None:
        x_ref = sky_image(Ny, Nx, seed)
    alpha = rng.normal(-0.7, 0.2, size=(Ny, Nx))
    nu = frequencies(L)
    return np.stack([x_ref * (nu[l] / nu[0]) ** alpha for l in range(L)])


def base_coverage(M: int, seed: int):
    """(om_y, om_x) = (v, u) ~ N(0, (pi/4)^2) clipped to [-pi, pi]."""
    rng = np.random.default_rng(seed + 104729)
    uv = rng.normal(0.0, np.pi / 4.0, size=(M, 2))
    uv = np.clip(uv, -np.pi, np.pi * (1.0 - 1e-12))
    return uv[:, 1].copy(), uv[:, 0].copy()


def channel_coverage(om_y, om_x, nu_l: float, nu_max: float):
    s = nu_l / nu_max
    return om_y * s, om_x * s


def split_blocks(M: int, n_blocks: int, rng) -> list:
    """Random block sizes (Dirichlet split) summing to M, each >= 1."""
    if n_blocks <= 1:
        return [M]
    w = rng.dirichlet(np.ones(n_blocks))
    sizes = np.maximum(1, np.floor(w * M).astype(int))
    sizes[-1] = M - int(np.sum(sizes[:-1]))
    if sizes[-1] < 1:
        sizes = np.full(n_blocks, M // n_blocks)
        sizes[-1] = M - int(np.sum(sizes[:-1]))
    return [int(s) for s in sizes]


def l2_bounds(block_sizes) -> list:
    Ml = float(sum(block_sizes))
    eps_l = np.sqrt(Ml + 2.0 * np.sqrt(Ml))
    return [float(np.sqrt(m / Ml) * eps_l) for m in block_sizes]


def noise(M: int, rng) -> np.ndarray:
    return (rng.standard_normal(M) + 1j * rng.standard_normal(M)) / np.sqrt(2.0)


def noise_sigma(y0: np.ndarray, snr_db: float) -> float:
    return float(10.0 ** (-snr_db / 20.0) * np.linalg.norm(y0) / np.sqrt(y0.size))


def jittered_splits(nchunks: int, N: int, jitter: float, rng) -> list:
    """Facet boundaries 0..N with sizes uniform in (1 +- jitter) x N/nchunks."""
    w = rng.uniform(1.0 - jitter, 1.0 + jitter, size=nchunks)
    edges = np.concatenate([[0.0], np.cumsum(w) / np.sum(w) * N])
    s = np.floor(edges + 0.5).astype(int)
    s[0], s[-1] = 0, N
    return [int(v) for v in s]
