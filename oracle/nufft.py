"""FP64 CPU restatement of the NUFFT measurement operator (oracle).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import this module, and only as the
checker.  The product path never calls it.

The reference builds its operator with ``op_p_nufft`` from the
``RI-measurement-operator`` submodule, which is not vendored
(``.gitmodules:1-6``; call site
``lib/operators/util_gen_measurement_operator_synth.m:86``:
``op_p_nufft([{v} {u}], [Ny Nx], [Ky Kx], [oy*Ny ox*Nx], [Ny/2 Nx/2], nW, [], 'minmax:kb')``).
This module restates the published method it implements:

  J. A. Fessler and B. P. Sutton, "Nonuniform fast Fourier transforms using
  min-max interpolation", IEEE TSP 51(2), 2003.

Conventions (parity against the MATLAB submodule is unpinned):

* image ``x`` is ``[Ny, Nx]`` (MATLAB dim 1 = y = rows, dim 2 = x = columns);
  the frequency pair of a visibility is ``(om_y, om_x) = (v, u)`` in radians;
* ``A(x) = fft2(s .* x, Ky_grid, Kx_grid)`` (zero padding at the end of each
  axis, unnormalised forward DFT), vectorised column-major (y fastest), as the
  reference's ``apply_scaled_fourier_transform.m:21-24`` expects;
* ``At(Y) = s .* crop(K * ifft2(Y))`` (the exact adjoint of ``A``);
* ``G`` maps the grid to visibilities: ``y_m = sum_k G[m,k] Y[k]`` approximates
  the NUDFT ``X(om) = sum_n x_n exp(-i om.(n - N/2))``;
* 1-D min-max coefficients for ``J`` neighbours ``k0+1..k0+J`` with
  ``k0 = floor(om/gamma - J/2)``, ``gamma = 2 pi / K``:
  ``g = (A^H A)^{-1} A^H b`` with ``A[n,j] = s_n exp(-i gamma (k0+j) n)`` and
  ``b_n = exp(-i om (n - N/2))`` (least-squares worst-case error, paper eq. 9);
* scaling factors ``s_n`` are a cosine series fitted to the reciprocal of the
  Kaiser-Bessel kernel's Fourier transform (``alpha = 2.34 J``, order 0), which
  makes every sum over ``n`` a Dirichlet kernel in closed form (paper
  section IV-C).  The fitted series *is* the scaling used (both here and on the
  GPU), so the operator is defined exactly by ``(N, K, J, a_l)``.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft
import scipy.sparse as sp
from scipy.special import i0

KB_ALPHA_PER_J = 2.34
N_COS_TERMS = 6  # highest cosine order L_c in the scaling series


def dirichlet(x, N, K):
    """D(x) = sum_{n=0}^{N-1} exp(-i*gamma*x*(n-c)), c=(N-1)/2, gamma=2pi/K.

    Closed form sin(pi*N*x/K)/sin(pi*x/K); equals N at x = 0.
    """
    x = np.asarray(x, dtype=np.float64)
    num = np.sin(np.pi * N * x / K)
    den = np.sin(np.pi * x / K)
    small = np.abs(den) < 1e-300
    out = np.where(small, float(N), num / np.where(small, 1.0, den))
    return out


def kb_ft(nu, J, alpha):
    """Fourier transform of the order-0 Kaiser-Bessel kernel of width J.

    kernel(k) = I0(alpha*sqrt(1-(2k/J)^2))/I0(alpha) for |k| <= J/2; its FT at
    frequency nu (cycles per grid sample) is
    J/I0(alpha) * sinh(sqrt(alpha^2-(pi J nu)^2)) / sqrt(alpha^2-(pi J nu)^2).
    """
    z2 = alpha ** 2 - (np.pi * J * np.asarray(nu, dtype=np.float64)) ** 2
    z = np.sqrt(np.abs(z2))
    with np.errstate(invalid="ignore", divide="ignore"):
        val = np.where(z2 > 0, np.sinh(z) / np.where(z > 0, z, 1.0),
                       np.where(z > 0, np.sin(z) / np.where(z > 0, z, 1.0), 1.0))
    return J / i0(alpha) * val


def scaling_cosine_coefs(N, K, J, n_terms=N_COS_TERMS):
    """Least-squares cosine-series fit of s_n = FT(0)/FT((n-c)/K).

    Returns a[0..n_terms] with s_n = sum_l a_l cos(2 pi l (n-c)/K).
    """
    alpha = KB_ALPHA_PER_J * J
    n = np.arange(N, dtype=np.float64)
    c = (N - 1) / 2.0
    target = kb_ft(0.0, J, alpha) / kb_ft((n - c) / K, J, alpha)
    basis = np.cos(2 * np.pi * np.outer(n - c, np.arange(n_terms + 1)) / K)
    a, *_ = np.linalg.lstsq(basis, target, rcond=None)
    return a


def scaling_factors(N, K, J, a=None):
    """The 1-D scaling factors s_n (n = 0..N-1) defined by the cosine series."""
    if a is None:
        a = scaling_cosine_coefs(N, K, J)
    n = np.arange(N, dtype=np.float64)
    c = (N - 1) / 2.0
    return np.cos(2 * np.pi * np.outer(n - c, np.arange(len(a))) / K) @ a


def _alpha_sym(a):
    """Two-sided coefficients alpha_l, l=-L..L, with alpha_{+-l} = a_l/2 (l>0)."""
    L = len(a) - 1
    al = np.zeros(2 * L + 1)
    al[L] = a[0]
    for l in range(1, L + 1):
        al[L + l] = al[L - l] = a[l] / 2.0
    return al, L


def minmax_R(N, K, J, a):
    """R[j,l] = S2(gamma*(j-l)), S2 the DTFT of s^2 about c (real, Toeplitz)."""
    al, L = _alpha_sym(a)
    ls = np.arange(-L, L + 1)
    d = np.subtract.outer(np.arange(J), np.arange(J)).astype(np.float64)
    R = np.zeros((J, J))
    for i1, l1 in enumerate(ls):
        for i2, l2 in enumerate(ls):
            R += al[i1] * al[i2] * dirichlet(d - (l1 + l2), N, K)
    return R


def minmax_T(N, K, J, a):
    return np.linalg.inv(minmax_R(N, K, J, a))


def minmax_r(dk, N, K, J, a):
    """r[m, j] = S(gamma*(dk_m - j)), j = 1..J (S: DTFT of s about c)."""
    al, L = _alpha_sym(a)
    dk = np.asarray(dk, dtype=np.float64)
    r = np.zeros(dk.shape + (J,))
    for j in range(1, J + 1):
        acc = np.zeros(dk.shape)
        for il, l in enumerate(range(-L, L + 1)):
            acc += al[il] * dirichlet(dk - j - l, N, K)
        r[..., j - 1] = acc
    return r


def interp_coefs_1d(om, N, K, J, a=None, T=None):
    """Min-max coefficients for one axis.

    Returns (k0, g) with grid neighbours (k0 + j) mod K, j = 1..J, and complex
    coefficients g[m, j-1] such that X(om) ~= sum_j g[m,j] Y[(k0+j) mod K].
    """
    if a is None:
        a = scaling_cosine_coefs(N, K, J)
    if T is None:
        T = minmax_T(N, K, J, a)
    om = np.asarray(om, dtype=np.float64)
    gam = 2 * np.pi / K
    k0 = np.floor(om / gam - J / 2.0).astype(np.int64)
    dk = om / gam - k0
    c = T @ minmax_r(dk, N, K, J, a).T            # [J, M]
    j = np.arange(1, J + 1, dtype=np.float64)[:, None]
    phase = np.pi / K * (((k0[None, :] + j.astype(np.int64)) * N) % (2 * K) + dk[None, :] - j)
    g = (np.exp(1j * phase) * c).T               # [M, J]
    return k0, dk, g


def build_G(om_y, om_x, Ny, Nx, Ky_grid, Kx_grid, Jy=7, Jx=7, weights=None):
    """Sparse interpolation matrix G (M x Ky_grid*Kx_grid), column-major grid index."""
    ay = scaling_cosine_coefs(Ny, Ky_grid, Jy)
    ax = scaling_cosine_coefs(Nx, Kx_grid, Jx)
    k0y, _, gy = interp_coefs_1d(om_y, Ny, Ky_grid, Jy, ay)
    k0x, _, gx = interp_coefs_1d(om_x, Nx, Kx_grid, Jx, ax)
    M = len(om_y)
    ky = (k0y[:, None] + np.arange(1, Jy + 1)[None, :]) % Ky_grid   # [M, Jy]
    kx = (k0x[:, None] + np.arange(1, Jx + 1)[None, :]) % Kx_grid   # [M, Jx]
    cols = (ky[:, :, None] + Ky_grid * kx[:, None, :]).reshape(M, Jy * Jx)
    vals = (gy[:, :, None] * gx[:, None, :]).reshape(M, Jy * Jx)
    if weights is not None:
        vals = vals * np.asarray(weights, dtype=np.float64)[:, None]
    rows = np.repeat(np.arange(M), Jy * Jx)
    return sp.csr_matrix((vals.ravel(), (rows, cols.ravel())), shape=(M, Ky_grid * Kx_grid))


class NufftOperator:
    """A / At / G for one image size; the per-channel G are built separately."""

    def __init__(self, Ny, Nx, oy=2, ox=2, Jy=7, Jx=7):
        self.Ny, self.Nx = Ny, Nx
        self.Ky, self.Kx = oy * Ny, ox * Nx
        self.Jy, self.Jx = Jy, Jx
        self.ay = scaling_cosine_coefs(Ny, self.Ky, Jy)
        self.ax = scaling_cosine_coefs(Nx, self.Kx, Jx)
        self.sy = scaling_factors(Ny, self.Ky, Jy, self.ay)
        self.sx = scaling_factors(Nx, self.Kx, Jx, self.ax)
        self.scale = np.outer(self.sy, self.sx)
        self.No = self.Ky * self.Kx

    def A(self, x):
        """x [Ny, Nx] real -> Fx (No,) complex, column-major vectorisation."""
        Y = sfft.fft2(self.scale * x, s=(self.Ky, self.Kx), workers=-1)
        return Y.reshape(-1, order="F")

    def At(self, Fx):
        """Fx (No,) complex -> [Ny, Nx] complex (exact adjoint of A)."""
        Y = np.asarray(Fx).reshape(self.Ky, self.Kx, order="F")
        x = sfft.ifft2(Y, workers=-1) * self.No
        return self.scale * x[: self.Ny, : self.Nx]

    def G(self, om_y, om_x, weights=None):
        return build_G(om_y, om_x, self.Ny, self.Nx, self.Ky, self.Kx,
                       self.Jy, self.Jx, weights)


def nudft(x, om_y, om_x):
    """Exact NUDFT X(om) = sum_n x[n] exp(-i om.(n - N/2)) (small sizes only)."""
    Ny, Nx = x.shape
    ny = np.arange(Ny) - Ny / 2.0
    nx = np.arange(Nx) - Nx / 2.0
    Ey = np.exp(-1j * np.outer(om_y, ny))   # [M, Ny]
    Ex = np.exp(-1j * np.outer(om_x, nx))   # [M, Nx]
    return np.einsum("my,yx,mx->m", Ey, x, Ex)


def coef_table(N, K, J, n_samples):
    """Complex table h[j, t] of the per-tap coefficient without the grid phase.

    g_j(om) = exp(i pi (k0+j) N / K) * h_j(dk) with dk = om/gamma - k0 in
    [J/2, J/2+1); the table samples dk = J/2 + t/n_samples, t = 0..n_samples.
    """
    a = scaling_cosine_coefs(N, K, J)
    T = minmax_T(N, K, J, a)
    dk = J / 2.0 + np.arange(n_samples + 1) / n_samples
    c = T @ minmax_r(dk, N, K, J, a).T   # [J, S]
    j = np.arange(1, J + 1)[:, None]
    return np.exp(1j * np.pi / K * (dk[None, :] - j)) * c
