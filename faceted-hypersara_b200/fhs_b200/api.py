"""Host-side mirror of the reference's MATLAB interface over the C ABI.

Function names, argument meaning and return values follow the reference
(basp-group/Faceted-HyperSARA):

* ``apply_direct_operator`` / ``apply_adjoint_operator``  (src/apply_*_operator.m:1)
* ``HS_forward_operator_G`` / ``HS_adjoint_operator_G``   (lib/operators/HS_*_operator_G.m:1)
* ``update_dual_data_fidelity``                           (src/update_dual_data_fidelity.m:1-6)
* ``proj_l2ball``, ``nuclear_norm``, ``compute_sara_prior`` (src/*.m:1)
* ``facetHyperSARA``, ``hyperSARA``, ``sara``              (src/{fhs,hs,sara}/*.m:1)

Image cubes are ``[Ny, Nx, L]`` float64 arrays (MATLAB order is used on the
wire: Fortran-contiguous copies are made as needed).  Visibilities and l2
bounds are nested lists ``y[l][b]`` / ``epsilon[l][b]`` as the reference's
cells.  The operator handle replaces the reference's ``A, At, G, W`` tuple.
Every computation runs in ``libfhs_b200.so`` on the GPU; a missing library or
device raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as LB
from ._lib import check, dptr, lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _cube_in(x, Ny, Nx):
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 2:
        x = x[:, :, None]
    if x.shape[:2] != (Ny, Nx):
        raise ValueError(f"expected [{Ny}, {Nx}, L] cube, got {x.shape}")
    return np.asfortranarray(x)


def _cplx_in(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.complex128)).view(np.float64)


class MeasurementOperator:
    """Phi_l = G_l A for every channel (op_p_nufft's A, At, G, W).

    ``om``: list over channels of (om_y, om_x) = (v, u) in radians;
    ``block_sizes``: list over channels of block sizes (defaults to 1 block);
    ``weights``: optional list over channels of per-visibility G row weights.
    """

    def __init__(self, Ny, Nx, om, block_sizes=None, weights=None, oy=2, ox=2, J=7, device=0):
        self.Ny, self.Nx, self.L = int(Ny), int(Nx), len(om)
        self.Ky, self.Kx = oy * Ny, ox * Nx
        self.No = self.Ky * self.Kx
        h = C.c_void_p()
        check(lib().fhs_measop_create(device, Ny, Nx, oy, ox, J, J, self.L, C.byref(h)))
        self._h = h
        self.device = device
        self.block_sizes = []
        try:
            for l, (omy, omx) in enumerate(om):
                omy, omx = _f64(omy), _f64(omx)
                M = omy.size
                bs = [M] if block_sizes is None else [int(b) for b in block_sizes[l]]
                self.block_sizes.append(bs)
                w = None if weights is None or weights[l] is None else _f64(weights[l])
                bsa = np.asarray(bs, dtype=np.int64)
                check(lib().fhs_measop_set_channel(h, l, M, dptr(omy), dptr(omx), dptr(w), len(bs),
                                                   bsa.ctypes.data_as(C.POINTER(C.c_int64))))
            check(lib().fhs_measop_commit(h))
        except Exception:
            lib().fhs_measop_destroy(h)
            self._h = None
            raise
        self.n_vis = [int(lib().fhs_measop_n_vis(h, l)) for l in range(self.L)]
        self.n_vis_total = int(sum(self.n_vis))

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().fhs_measop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- A / At ----------------------------------------------------------
    def A(self, x):
        """Scaled zero-padded FFT of one image -> Fx (No,) complex."""
        x = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(self.Ny, self.Nx))
        out = np.empty(self.No, dtype=np.complex128)
        check(lib().fhs_scaled_fft(self._h, dptr(x.reshape(-1, order="F")), dptr(out.view(np.float64))))
        return out

    def At(self, Fx):
        """Adjoint of A: Fx (No,) -> [Ny, Nx] complex."""
        Fx = _cplx_in(Fx)
        out = np.empty(self.Ny * self.Nx, dtype=np.complex128)
        check(lib().fhs_scaled_fft_adjoint(self._h, dptr(Fx), dptr(out.view(np.float64))))
        return out.reshape(self.Ny, self.Nx, order="F")

    # -- blocks of one channel ---------------------------------------------
    def split(self, l, v):
        out, pos = [], 0
        for m in self.block_sizes[l]:
            out.append(v[pos:pos + m])
            pos += m
        return out

    def flatten(self, yl):
        return np.concatenate([np.asarray(b, dtype=np.complex128).ravel() for b in yl]) if len(yl) else \
            np.zeros(0, np.complex128)

    def operator_norm(self, max_iter=200, tol=1e-8):
        out = np.empty(self.L)
        check(lib().fhs_operator_norm(self._h, max_iter, tol, dptr(out)))
        return out


# ------------------------------------------------------------------ functions
def apply_direct_operator(Fx, op: MeasurementOperator, channel: int = 0):
    """src/apply_direct_operator.m:1 (Lambda = 1): y = G Fx, blocks concatenated."""
    Fx = _cplx_in(Fx)
    y = np.empty(op.n_vis[channel], dtype=np.complex128)
    check(lib().fhs_apply_direct_operator(op.handle, channel, dptr(Fx), dptr(y.view(np.float64))))
    return y


def apply_adjoint_operator(y, op: MeasurementOperator, channel: int = 0):
    """src/apply_adjoint_operator.m:1 (Lambda = 1): Fx = G' y."""
    y = _cplx_in(y)
    Fx = np.empty(op.No, dtype=np.complex128)
    check(lib().fhs_apply_adjoint_operator(op.handle, channel, dptr(y), dptr(Fx.view(np.float64))))
    return Fx


def HS_forward_operator_G(x, op: MeasurementOperator):
    """lib/operators/HS_forward_operator_G.m:36-52 -> y[l][b]."""
    x = _cube_in(x, op.Ny, op.Nx)
    y = np.empty(op.n_vis_total, dtype=np.complex128)
    check(lib().fhs_forward_operator(op.handle, dptr(x.reshape(-1, order="F")), dptr(y.view(np.float64))))
    out, pos = [], 0
    for l in range(op.L):
        out.append(op.split(l, y[pos:pos + op.n_vis[l]]))
        pos += op.n_vis[l]
    return out


def HS_adjoint_operator_G(y, op: MeasurementOperator):
    """lib/operators/HS_adjoint_operator_G.m:42-57, real part -> [Ny, Nx, L]."""
    flat = np.concatenate([op.flatten(yl) for yl in y])
    flat = _cplx_in(flat)
    x = np.empty(op.Ny * op.Nx * op.L)
    check(lib().fhs_adjoint_operator(op.handle, dptr(flat), dptr(x)))
    return x.reshape(op.Ny, op.Nx, op.L, order="F")
