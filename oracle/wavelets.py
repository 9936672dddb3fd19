"""FP64 CPU restatement of the SARA dictionary (oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/nufft.py``).

The reference takes the SARA dictionary from the ``SARA-dictionary``
submodule (not vendored, ``.gitmodules:1-6``): ``op_p_sp_wlt_basis`` for the
SARA solver (``imaging/imaging.m:802``) and ``sdwt2_sara_faceting`` /
``isdwt2_sara_faceting`` for the faceted solver
(``src/fhs/fhs_update_dual_sparsity.m:75,92``), with MATLAB's Wavelet Toolbox in
zero-padding mode (``dwtmode('zpd')``, ``imaging/imaging.m:801``).  This module
restates:

* Daubechies extremal-phase orthonormal filters db1..db8 by spectral
  factorisation (I. Daubechies, *Ten Lectures on Wavelets*, 1992, sec. 6.1),
  oriented as MATLAB's reconstruction low-pass ``Lo_R`` (largest taps first);
  ``Lo_D = reverse(Lo_R)``, ``Hi_R[k] = (-1)^k Lo_R[L-1-k]``,
  ``Hi_D = reverse(Hi_R)``;
* the zero-padded one-level DWT: full convolution then keep the odd samples,
  ``out[p] = sum_t f[t] x[2p+1-t]``, ``p < floor((n+L-1)/2)``;
* ``dwt2`` filtering dim 2 then dim 1 with subbands
  ``a = lo2.lo1, h = lo2.hi1, v = hi2.lo1, d = hi2.hi1``;
* ``wavedec2`` coefficient vector ``[A_J H_J V_J D_J ... H_1 V_1 D_1]``,
  each subband vectorised column-major;
* the SARA analysis ``Psit(x) = [wavedec2(x, db1..db8), x(:)] / sqrt(9)`` and
  synthesis ``Psi`` = its adjoint (``nu1 = 1`` in ``imaging/imaging.m:845``
  states that Psi is a Parseval frame).

With zero padding and orthonormal filters every level is an isometry, so the
multilevel transform is an isometry and ``waverec2`` equals its adjoint.  The
faceted transform ``sdwt2`` of the faceted solver produces, by construction
(Prusa 2012, segmentwise DWT), the same coefficient set as the global
transform, split over facets; the oracle uses the global one.
"""
from __future__ import annotations

from math import comb

import numpy as np

from ._par import pmap

SARA_WAVELETS = ("db1", "db2", "db3", "db4", "db5", "db6", "db7", "db8")
N_BASES = len(SARA_WAVELETS) + 1   # + Dirac ("self")


def daubechies_lo_r(p: int) -> np.ndarray:
    """Extremal-phase Daubechies scaling filter with p vanishing moments.

    H(z) = sqrt(2) ((1+z^-1)/2)^p Q(z^-1), |Q|^2 = P(sin^2(w/2)) with
    P(y) = sum_{k<p} C(p-1+k, k) y^k; the roots of Q are the ones inside the
    unit circle of z^{p-1} P((2 - z - 1/z)/4).
    """
    if p == 1:
        return np.array([1.0, 1.0]) / np.sqrt(2.0)
    # polynomial in y, then substitute y = (2 - z - 1/z)/4 and multiply z^{p-1}
    Py = [comb(p - 1 + k, k) for k in range(p)]
    # (2 - z - 1/z)/4 * z = (-z^2 + 2z - 1)/4 -> y^k z^k = ((-z^2+2z-1)/4)^k
    base = np.array([-0.25, 0.5, -0.25])   # coefficients of z^2, z, 1
    poly = np.zeros(2 * p - 1)             # degree 2(p-1) in z, highest first
    for k, ck in enumerate(Py):
        term = np.array([1.0])
        for _ in range(k):
            term = np.convolve(term, base)
        # term has degree 2k; multiply by z^{p-1-k}
        term = np.concatenate([term, np.zeros(p - 1 - k)])
        poly[len(poly) - len(term):] += ck * term
    roots = np.roots(poly)
    inside = roots[np.abs(roots) < 1.0]
    q = np.real(np.poly(inside))               # prod (z - r), highest first
    h = q
    for _ in range(p):
        h = np.convolve(h, [1.0, 1.0])
    h = h / np.sum(h) * np.sqrt(2.0)
    return h


def wavelet_filters(name: str):
    """(Lo_D, Hi_D, Lo_R, Hi_R) in MATLAB's orientation."""
    p = int(name[2:])
    lo_r = daubechies_lo_r(p)
    L = len(lo_r)
    k = np.arange(L)
    hi_r = ((-1.0) ** k) * lo_r[::-1]
    return lo_r[::-1].copy(), hi_r[::-1].copy(), lo_r, hi_r


def dwt_len(n: int, L: int) -> int:
    return (n + L - 1) // 2


def dwt_axis(x: np.ndarray, f: np.ndarray, axis: int) -> np.ndarray:
    """out[p] = sum_t f[t] x[2p+1-t] along ``axis`` (x zero outside)."""
    x = np.moveaxis(x, axis, -1)
    n = x.shape[-1]
    L = len(f)
    m = dwt_len(n, L)
    xp = np.zeros(x.shape[:-1] + (n + 2 * L + 2,), dtype=x.dtype)
    xp[..., L:L + n] = x
    out = np.zeros(x.shape[:-1] + (m,), dtype=np.result_type(x, f))
    for t in range(L):
        # x[2p+1-t] -> xp[2p+1-t+L]
        start = 1 - t + L
        out += f[t] * xp[..., start:start + 2 * m:2]
    return np.moveaxis(out, -1, axis)


def idwt_axis(c: np.ndarray, f: np.ndarray, n: int, axis: int) -> np.ndarray:
    """Adjoint of ``dwt_axis``: x[i] = sum_p c[p] f[2p+1-i], i < n."""
    c = np.moveaxis(c, axis, -1)
    m = c.shape[-1]
    L = len(f)
    u = np.zeros(c.shape[:-1] + (2 * m + 2 * L + n + 2,), dtype=c.dtype)
    u[..., 1:2 * m:2] = c            # u[2p+1] = c[p]
    out = np.zeros(c.shape[:-1] + (n,), dtype=np.result_type(c, f))
    for t in range(L):
        # x[i] += f[t] * u[i + t]
        out += f[t] * u[..., t:t + n]
    return np.moveaxis(out, -1, axis)


def level_sizes(n0: int, n1: int, L: int, nlevel: int):
    sizes = []
    for _ in range(nlevel):
        n0, n1 = dwt_len(n0, L), dwt_len(n1, L)
        sizes.append((n0, n1))
    return sizes


def n_coefs_basis(n0: int, n1: int, L: int, nlevel: int) -> int:
    sizes = level_sizes(n0, n1, L, nlevel)
    return sizes[-1][0] * sizes[-1][1] + 3 * sum(a * b for a, b in sizes)


def n_coefs_sara(n0: int, n1: int, nlevel: int = 4) -> int:
    return sum(n_coefs_basis(n0, n1, 2 * p, nlevel) for p in range(1, 9)) + n0 * n1


def _vec(a):
    """Column-major vectorisation of the last two axes -> [..., n0*n1]."""
    return np.swapaxes(a, -1, -2).reshape(a.shape[:-2] + (-1,))


def _unvec(v, n0, n1):
    return np.swapaxes(v.reshape(v.shape[:-1] + (n1, n0)), -1, -2)


def wavedec2(x: np.ndarray, nlevel: int, name: str) -> np.ndarray:
    """x [..., n0, n1] -> coefficient vector [..., s] (MATLAB wavedec2 layout)."""
    lo_d, hi_d, _, _ = wavelet_filters(name)
    a = x
    details = []
    for _ in range(nlevel):
        lo2 = dwt_axis(a, lo_d, -1)
        hi2 = dwt_axis(a, hi_d, -1)
        a_n = dwt_axis(lo2, lo_d, -2)
        h = dwt_axis(lo2, hi_d, -2)
        v = dwt_axis(hi2, lo_d, -2)
        d = dwt_axis(hi2, hi_d, -2)
        details.append((h, v, d))
        a = a_n
    parts = [_vec(a)]
    for h, v, d in reversed(details):
        parts += [_vec(h), _vec(v), _vec(d)]
    return np.concatenate(parts, axis=-1)


def waverec2(c: np.ndarray, n0: int, n1: int, nlevel: int, name: str) -> np.ndarray:
    """Adjoint (= inverse on the range) of ``wavedec2``."""
    lo_d, hi_d, _, _ = wavelet_filters(name)
    L = len(lo_d)
    sizes = [(n0, n1)] + level_sizes(n0, n1, L, nlevel)
    pos = 0
    m0, m1 = sizes[-1]
    a = _unvec(c[..., pos:pos + m0 * m1], m0, m1)
    pos += m0 * m1
    for lev in range(nlevel, 0, -1):
        m0, m1 = sizes[lev]
        sub = []
        for _ in range(3):
            sub.append(_unvec(c[..., pos:pos + m0 * m1], m0, m1))
            pos += m0 * m1
        h, v, d = sub
        p0, p1 = sizes[lev - 1]
        lo2 = idwt_axis(a, lo_d, p0, -2) + idwt_axis(h, hi_d, p0, -2)
        hi2 = idwt_axis(v, lo_d, p0, -2) + idwt_axis(d, hi_d, p0, -2)
        a = idwt_axis(lo2, lo_d, p1, -1) + idwt_axis(hi2, hi_d, p1, -1)
    return a


def _channel_chunks(lead, plane=None, min_elems=1 << 19):
    """Slices of the leading (channel) axis for threaded SARA transforms, or
    None to run sequentially (small transforms: thread overhead dominates)."""
    if len(lead) != 1:
        return None
    L = lead[0]
    if plane is not None and L * plane < min_elems:
        return None
    from ._par import n_threads
    k = max(1, min(L, n_threads() // 2))
    edges = [round(i * L / k) for i in range(k + 1)]
    return [slice(a, b) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def sara_analysis(x: np.ndarray, nlevel: int = 4) -> np.ndarray:
    """Psit: x [..., n0, n1] -> [..., s], s = n_coefs_sara(n0, n1, nlevel)."""
    chunks = _channel_chunks(x.shape[:-2], x.shape[-2] * x.shape[-1])
    if chunks is None:
        parts = [wavedec2(x, nlevel, w) for w in SARA_WAVELETS]
    else:   # (basis, channel chunk) jobs on the oracle's threads
        jobs = [(w, c) for w in SARA_WAVELETS for c in chunks]
        res = pmap(lambda j: wavedec2(x[j[1]], nlevel, j[0]), jobs)
        parts = [np.concatenate(res[i * len(chunks):(i + 1) * len(chunks)], axis=0)
                 for i in range(len(SARA_WAVELETS))]
    parts.append(_vec(x))
    return np.concatenate(parts, axis=-1) / np.sqrt(N_BASES)


def sara_synthesis(c: np.ndarray, n0: int, n1: int, nlevel: int = 4) -> np.ndarray:
    """Psi: [..., s] -> [..., n0, n1] (adjoint of ``sara_analysis``)."""
    jobs, pos = [], 0
    for w in SARA_WAVELETS:
        sb = n_coefs_basis(n0, n1, 2 * int(w[2:]), nlevel)
        jobs.append((w, pos, sb))
        pos += sb
    chunks = _channel_chunks(c.shape[:-1], n0 * n1)
    if chunks is None:
        recs = [waverec2(c[..., p0:p0 + sb], n0, n1, nlevel, w) for w, p0, sb in jobs]
    else:   # (basis, channel chunk) jobs on the oracle's threads
        res = pmap(lambda j: waverec2(c[j[1]][..., j[0][1]:j[0][1] + j[0][2]], n0, n1, nlevel, j[0][0]),
                   [(b, ch) for b in jobs for ch in chunks])
        recs = [np.concatenate(res[i * len(chunks):(i + 1) * len(chunks)], axis=0) for i in range(len(jobs))]
    out = 0.0
    for r in recs:   # summed in basis order, as the sequential form
        out = out + r
    out = out + _unvec(c[..., pos:pos + n0 * n1], n0, n1)
    return out / np.sqrt(N_BASES)


def sara_basis_ranges(n0: int, n1: int, nlevel: int = 4):
    """[(start, stop)] of each basis inside the SARA vector (db1..db8, Dirac)."""
    out, pos = [], 0
    for p in range(1, 9):
        sb = n_coefs_basis(n0, n1, 2 * p, nlevel)
        out.append((pos, pos + sb))
        pos += sb
    out.append((pos, pos + n0 * n1))
    return out
