"""Small synthetic problems for the oracle (test infrastructure only).

Builds a :class:`oracle.solvers.DataTerm` from the seeded generators of the
product package (inputs only; every operator here is the oracle's own).
"""
from __future__ import annotations

import numpy as np

from ._par import pmap
from .nufft import NufftOperator
from .solvers import DataTerm


def make_problem(Ny, Nx, L, M_per_channel, n_blocks, seed, snr_db=40.0, synth=None):
    """Return (data, x_true, meta) with whitened G/y and chi2 l2 bounds.

    ``M_per_channel``: int or list of ints; ``n_blocks``: int or list of ints.
    meta holds the per-channel coverage (om_y, om_x), block sizes, sigma.
    """
    if synth is None:
        raise ValueError("pass the synth module")
    op = NufftOperator(Ny, Nx)
    x = synth.sky_cube(Ny, Nx, L, seed) if L > 1 else synth.sky_image(Ny, Nx, seed)[None]
    Ms = [M_per_channel] * L if np.isscalar(M_per_channel) else list(M_per_channel)
    nbs = [n_blocks] * L if np.isscalar(n_blocks) else list(n_blocks)
    om_y0, om_x0 = synth.base_coverage(max(Ms), seed)
    nu = synth.frequencies(L)
    rng = np.random.default_rng(seed + 31)
    G_all, y_all, eps_all, meta = [], [], [], {"om": [], "blocks": [], "sigma": []}

    def build(l):   # no random draws here: the seeded stream below stays in channel order
        oy, ox = synth.channel_coverage(om_y0[: Ms[l]], om_x0[: Ms[l]], nu[l], nu[-1])
        G = op.G(oy, ox)
        return oy, ox, G, G @ op.A(x[l])
    built = pmap(build, range(L))
    for l in range(L):
        oy, ox, G, y0 = built[l]
        built[l] = None   # large sizes: hold one channel's full G at a time besides the blocks
        sizes = synth.split_blocks(Ms[l], nbs[l], rng)
        sigma = synth.noise_sigma(y0, snr_db)
        yl = (y0 + sigma * synth.noise(Ms[l], rng)) / sigma
        G.data /= sigma   # whitening, in place
        Gb, yb = [], []
        pos = 0
        for m in sizes:
            Gb.append(G[pos:pos + m] if len(sizes) > 1 else G)
            yb.append(yl[pos:pos + m])
            pos += m
        del G
        G_all.append(Gb)
        y_all.append(yb)
        eps_all.append(synth.l2_bounds(sizes))
        meta["om"].append((oy, ox))
        meta["blocks"].append(sizes)
        meta["sigma"].append(sigma)
    return DataTerm(op, G_all, y_all, eps_all), x, meta
