"""Facet geometry and apodisation windows (oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/nufft.py``).

``split_range`` and ``generate_weights`` live in the missing ``SARA-dictionary``
submodule; their call sites fix what they must return:

* ``src/fhs/facetHyperSARA.m:296-321``: base facets from
  ``split_range(Q, N)`` (contiguous 1-based inclusive ranges) and nuclear-norm
  facets from ``split_range(Q, N, overlap)``, whose ranges extend the base
  range towards lower indices by ``overlap`` pixels (``fhs_setup_priors.m:157``
  and the ``x_facet(overlap+1:end, ...)`` writes at
  ``facetHyperSARA.m:727``);
* ``src/fhs/fhs_setup_priors.m:189``: ``w{q} = generate_weights(qx, qy, Qx, Qy,
  window_type, dims, dims_o, overlap_size)`` of size ``dims_o``; default window
  ``'triangular'`` (``imaging/imaging.m:210``).

Restated here (unpinned): ``split_range`` rounds ``linspace(0, N, Q+1)`` half
away from zero; the triangular window is the separable product of 1-D ramps
that rise over the facet's own overlap and fall over the next facet's overlap,
so the windows of all facets sum to one at every pixel.
"""
from __future__ import annotations

import numpy as np


def split_range(nchunks: int, N: int, overlap: int = 0, splits=None):
    """0-based half-open ranges [(start, stop)] of nchunks contiguous facets.

    ``splits`` (length nchunks+1, 0..N) overrides the uniform split (used for
    uneven facets).  With ``overlap`` > 0 every facet but the first starts
    ``overlap`` pixels earlier (clipped at 0).
    """
    if splits is None:
        splits = np.floor(np.linspace(0, N, nchunks + 1) + 0.5).astype(int)
    rg = []
    for q in range(nchunks):
        a, b = int(splits[q]), int(splits[q + 1])
        if q > 0 and overlap > 0:
            a = max(a - overlap, 0)
        rg.append((a, b))
    return rg


def jittered_splits(nchunks: int, N: int, jitter: float, rng) -> np.ndarray:
    """Facet boundaries with sizes uniform(1-jitter, 1+jitter) x N/nchunks."""
    w = rng.uniform(1.0 - jitter, 1.0 + jitter, size=nchunks)
    edges = np.concatenate([[0.0], np.cumsum(w) / np.sum(w) * N])
    s = np.floor(edges + 0.5).astype(int)
    s[0], s[-1] = 0, N
    return s


def window_1d(q: int, rg_base, rg_over, window_type: str = "triangular") -> np.ndarray:
    a, b = rg_over[q]
    n = b - a
    w = np.ones(n)
    if window_type in ("none", "ones"):
        return w
    if window_type != "triangular":
        raise ValueError(f"unsupported window {window_type}")
    o_left = rg_base[q][0] - rg_over[q][0]
    if o_left > 0:
        w[:o_left] = (np.arange(o_left) + 1.0) / (o_left + 1.0)
    if q + 1 < len(rg_base):
        o_right = rg_base[q + 1][0] - rg_over[q + 1][0]
        if o_right > 0:
            w[n - o_right:] *= 1.0 - (np.arange(o_right) + 1.0) / (o_right + 1.0)
    return w


class FacetGeometry:
    """Qy x Qx nuclear-norm facets; facet index q = qx*Qy + qy (y fastest)."""

    def __init__(self, Ny, Nx, Qy, Qx, overlap=(0, 0), splits_y=None, splits_x=None,
                 window_type="triangular"):
        self.Ny, self.Nx, self.Qy, self.Qx = Ny, Nx, Qy, Qx
        self.base_y = split_range(Qy, Ny, 0, splits_y)
        self.base_x = split_range(Qx, Nx, 0, splits_x)
        self.over_y = split_range(Qy, Ny, overlap[0], splits_y)
        self.over_x = split_range(Qx, Nx, overlap[1], splits_x)
        self.wy = [window_1d(q, self.base_y, self.over_y, window_type) for q in range(Qy)]
        self.wx = [window_1d(q, self.base_x, self.over_x, window_type) for q in range(Qx)]
        self.Q = Qy * Qx

    def facets(self):
        """Yield (q, (y0, y1), (x0, x1), window[ny, nx]) over overlapped facets."""
        for qx in range(self.Qx):
            for qy in range(self.Qy):
                yield (qx * self.Qy + qy, self.over_y[qy], self.over_x[qx],
                       np.outer(self.wy[qy], self.wx[qx]))

    def n_pixels(self, q):
        qx, qy = divmod(q, self.Qy)
        (a, b), (c, d) = self.over_y[qy], self.over_x[qx]
        return (b - a) * (d - c)
