"""Host-side mirror of the reference's MATLAB interface over the C ABI.

Function names, argument meaning and return values follow the reference
(basp-group/Faceted-HyperSARA):

* ``apply_direct_operator`` / ``apply_adjoint_operator``  (src/apply_*_operator.m:1)
* ``HS_forward_operator_G`` / ``HS_adjoint_operator_G``   (lib/operators/HS_*_operator_G.m:1)
* ``update_dual_data_fidelity`` (pU = 1) and ``update_dual_data_fidelity_precond``
                                                          (src/update_dual_data_fidelity.m:1-6)
* ``HS_forward_operator_precond_G`` / ``HS_adjoint_operator_precond_G``,
  ``gen_preconditioning_matrix``                          (lib/operators/, util_gen_preconditioning_matrix)
* ``proj_l2ball``, ``nuclear_norm``, ``compute_sara_prior`` (src/*.m:1)
* ``facetHyperSARA``, ``hyperSARA``, ``sara``              (src/{fhs,hs,sara}/*.m:1)
* ``MeasurementOperator.dimensionality_reduction`` / ``reduce_data``
                    (lib/operators/util_load_data_gen_dr_measurement_operator.m)

Image cubes are ``[Ny, Nx, L]`` float64 arrays (MATLAB order is used on the
wire: Fortran-contiguous copies are made as needed).  Visibilities and l2
bounds are nested lists ``y[l][b]`` / ``epsilon[l][b]`` as the reference's
cells.  The operator handle replaces the reference's ``A, At, G, W`` tuple
(and ``Lambda`` for a visibility-gridding operator).
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

    @classmethod
    def _from_dr_handle(cls, h, vis):
        self = cls.__new__(cls)
        self._h = h
        self.Ny, self.Nx, self.L = vis.Ny, vis.Nx, vis.L
        self.Ky, self.Kx, self.No = vis.Ky, vis.Kx, vis.No
        self.device = vis.device
        self.n_vis = [int(lib().fhs_measop_n_vis(h, l)) for l in range(self.L)]
        self.n_vis_total = int(sum(self.n_vis))
        self.block_sizes = [[n] for n in self.n_vis]
        self.W, self.Lambda = [], []
        for l, n in enumerate(self.n_vis):
            cells = np.empty(n, dtype=np.int64)
            lam = np.empty(n)
            check(lib().fhs_measop_dr_cells(h, l, cells.ctypes.data_as(C.POINTER(C.c_int64))))
            check(lib().fhs_measop_dr_lambda(h, l, dptr(lam)))
            self.W.append(cells)
            self.Lambda.append(lam)
        return self

    @property
    def handle(self):
        return self._h

    @property
    def is_dr(self):
        return bool(lib().fhs_measop_is_dr(self._h) == 1)

    def dimensionality_reduction(self):
        """lib/operators/util_load_data_gen_dr_measurement_operator.m:109-228:
        the visibility-gridding operator of this one (H = G'G over each
        channel's blocks, W = diag(H) > 0, Lambda = diag(H)^-1/2, one block per
        channel).  Returns a MeasurementOperator whose data entries of channel
        l are the active cells ``W[l]`` (0-based column-major grid indices,
        ascending) with weights ``Lambda[l]``; the operator functions, the
        dual update and the solvers take it in place of this one."""
        h = C.c_void_p()
        check(lib().fhs_measop_create_dr(self._h, C.byref(h)))
        return MeasurementOperator._from_dr_handle(h, self)

    def reduce_data(self, dr, y):
        """Lambda .* (G' y)(W) per channel (util_load_data_gen_dr_measurement_
        operator.m:180, 219): the gridded data of visibilities ``y[l]`` (one
        array or a list of blocks per channel) for the DR operator ``dr`` made
        from this operator, as ``[[y_dr_l]]``.  Applied to a noise draw it
        gives the gridded noise whose norm is the DR l2 bound (:184-201, 226)."""
        out = []
        for l in range(self.L):
            yl = y[l]
            v = self.flatten(yl) if isinstance(yl, (list, tuple)) else np.asarray(yl, dtype=np.complex128)
            g = apply_adjoint_operator(v, self, l)
            out.append([dr.Lambda[l] * g[dr.W[l]]])
        return out

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

    def operator_norm(self, max_iter=200, tol=1e-8, precond=False):
        """Per-channel squared norms of G_l A (precond: of sqrt(pU) G_l A),
        lib/utils/util_operator_norm.m:43-61."""
        out = np.empty(self.L)
        fn = lib().fhs_operator_norm_precond if precond else lib().fhs_operator_norm
        check(fn(self._h, max_iter, tol, dptr(out)))
        return out

    def autotune(self):
        """Time the launch-shape candidates (FFT planes per launch, gridding
        work-item size) on this operator and keep the fastest; returns the
        record of ``tuning()``."""
        t = LB.Tuning()
        check(lib().fhs_measop_autotune(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, fft_chunk, grid_slice):
        """Fix the launch shapes without measuring (fft_chunk 0: all planes)."""
        check(lib().fhs_measop_set_tuning(self._h, int(fft_chunk), int(grid_slice)))

    def tuning(self):
        """The shapes in use and the autotuner's measurements (ms per candidate)."""
        t = LB.Tuning()
        check(lib().fhs_measop_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_preconditioner(self, pU):
        """Attach aW: ``pU[l]`` is one channel's preconditioner, either one
        array over its visibilities or a list over its blocks."""
        if len(pU) != self.L:
            raise ValueError(f"expected {self.L} channels of preconditioner")
        for l, pl in enumerate(pU):
            a = _f64(np.concatenate([np.asarray(b, dtype=np.float64).ravel() for b in pl])
                     if isinstance(pl, (list, tuple)) else np.asarray(pl, dtype=np.float64).ravel())
            if a.size != self.n_vis[l]:
                raise ValueError(f"channel {l}: expected {self.n_vis[l]} preconditioner entries, got {a.size}")
            check(lib().fhs_measop_set_preconditioner(self._h, l, dptr(a)))


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


def HS_forward_operator_precond_G(x, op: MeasurementOperator):
    """lib/operators/HS_forward_operator_precond_G.m:40-55: sqrt(aW) .* G A x -> y[l][b]."""
    x = _cube_in(x, op.Ny, op.Nx)
    y = np.empty(op.n_vis_total, dtype=np.complex128)
    check(lib().fhs_forward_operator_precond(op.handle, dptr(x.reshape(-1, order="F")),
                                             dptr(y.view(np.float64))))
    out, pos = [], 0
    for l in range(op.L):
        out.append(op.split(l, y[pos:pos + op.n_vis[l]]))
        pos += op.n_vis[l]
    return out


def HS_adjoint_operator_precond_G(y, op: MeasurementOperator):
    """lib/operators/HS_adjoint_operator_precond_G.m: real(At(G' (sqrt(aW) .* y))) -> [Ny, Nx, L]."""
    flat = _cplx_in(np.concatenate([op.flatten(yl) for yl in y]))
    x = np.empty(op.Ny * op.Nx * op.L)
    check(lib().fhs_adjoint_operator_precond(op.handle, dptr(flat), dptr(x)))
    return x.reshape(op.Ny, op.Nx, op.L, order="F")


def gen_preconditioning_matrix(om_y, om_x, Ky, Kx, sub_pixels=1):
    """util_gen_preconditioning_matrix with gen_uniform_weight_matrix = true:
    pU = 1 / (visibilities in the same cell of a (Ky sub) x (Kx sub) grid)."""
    omy, omx = _f64(om_y).ravel(), _f64(om_x).ravel()
    if omy.size != omx.size:
        raise ValueError("om_y and om_x differ in length")
    out = np.empty(omy.size)
    check(lib().fhs_gen_preconditioning_matrix(omy.size, dptr(omy), dptr(omx), int(Ky), int(Kx),
                                               int(sub_pixels), dptr(out)))
    return out


def compute_residual_images(x, y, op: MeasurementOperator):
    """src/compute_residual_images.m:83-102 (DR operator: :42-80): PSF-normalised
    residual images real(At(G'(y - G A x))) -> [Ny, Nx, L]."""
    xc = _cube_in(x, op.Ny, op.Nx)
    yf = _cplx_in(np.concatenate([op.flatten(v) for v in y]))
    out = np.empty(op.Ny * op.Nx * op.L)
    check(lib().fhs_compute_residual_images(op.handle, dptr(yf), dptr(xc.reshape(-1, order="F")), dptr(out)))
    return out.reshape(op.Ny, op.Nx, op.L, order="F")


def proj_l2ball(x, eps, y, device: int = 0):
    """src/proj_l2ball.m:20-22 on the GPU (FP64)."""
    x = np.asarray(x)
    cplx = np.iscomplexobj(x) or np.iscomplexobj(y)
    xa = _cplx_in(np.asarray(x, dtype=np.complex128).ravel())
    ya = _cplx_in(np.asarray(y, dtype=np.complex128).ravel())
    p = np.empty(x.size, dtype=np.complex128)
    check(lib().fhs_proj_l2ball(device, x.size, dptr(xa), float(eps), dptr(ya), dptr(p.view(np.float64))))
    p = p.reshape(x.shape)
    return p if cplx else p.real.copy()


def nuclear_norm(x, device: int = 0):
    """src/nuclear_norm.m:25-26: x [Ny, Nx, L] (or [N, L])."""
    x = np.asarray(x, dtype=np.float64)
    L = x.shape[-1]
    xm = np.asfortranarray(x.reshape(-1, L, order="F"))
    f = np.zeros(1)
    check(lib().fhs_nuclear_norm(device, xm.shape[0], L, dptr(xm.reshape(-1, order="F")), dptr(f)))
    return float(f[0])


def sara_n_coefs(Ny, Nx, nlevel=4):
    return int(lib().fhs_sara_n_coefs(Ny, Nx, nlevel))


def sara_analysis(x, nlevel=4, device: int = 0):
    """SARA Psit (op_p_sp_wlt_basis): x [Ny, Nx, L] -> coefficients [s, L]."""
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 2:
        x = x[:, :, None]
    Ny, Nx, L = x.shape
    s = sara_n_coefs(Ny, Nx, nlevel)
    xf = np.asfortranarray(x)
    out = np.empty((s, L), order="F")
    check(lib().fhs_sara_analysis(device, Ny, Nx, L, nlevel, dptr(xf.reshape(-1, order="F")),
                                  dptr(out.reshape(-1, order="F"))))
    return out


def sara_synthesis(c, Ny, Nx, nlevel=4, device: int = 0):
    """SARA Psi: coefficients [s, L] -> [Ny, Nx, L]."""
    c = np.asarray(c, dtype=np.float64)
    if c.ndim == 1:
        c = c[:, None]
    L = c.shape[1]
    cf = np.asfortranarray(c)
    out = np.empty((Ny, Nx, L), order="F")
    check(lib().fhs_sara_synthesis(device, Ny, Nx, L, nlevel, dptr(cf.reshape(-1, order="F")),
                                   dptr(out.reshape(-1, order="F"))))
    return out


def compute_sara_prior(x, nlevel=4, device: int = 0):
    """src/compute_sara_prior.m:35-41: ||Psit X||_{2,1}."""
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 2:
        x = x[:, :, None]
    Ny, Nx, L = x.shape
    xf = np.asfortranarray(x)
    f = np.zeros(1)
    check(lib().fhs_compute_sara_prior(device, Ny, Nx, L, nlevel, dptr(xf.reshape(-1, order="F")), dptr(f)))
    return float(f[0])


def update_dual_data_fidelity(v2, y, x, Fx_old, op: MeasurementOperator, epsilon, sigma22):
    """src/update_dual_data_fidelity.m:1-6 with pU = 1 (a DR operator takes the
    flag_dimensionality_reduction branch, :85-125).

    Returns (v2, Ftx, Fx_old, norm_res, global_norm_res, norm_epsilon) with the
    reference's meaning (v2/norm_res as nested lists, Fx_old [No, L])."""
    xc = _cube_in(x, op.Ny, op.Nx)
    v2f = _cplx_in(np.concatenate([op.flatten(v) for v in v2])).copy()
    yf = _cplx_in(np.concatenate([op.flatten(v) for v in y]))
    Fo = np.asfortranarray(np.asarray(Fx_old, dtype=np.complex128).reshape(op.No, op.L, order="F"))
    Fo_flat = np.ascontiguousarray(Fo.T).view(np.float64).copy()   # channel after channel
    eps = np.concatenate([np.asarray(e, dtype=np.float64).ravel() for e in epsilon])
    s22 = _f64(np.broadcast_to(np.asarray(sigma22, dtype=np.float64), (op.L,)))
    Ftx = np.empty(op.Ny * op.Nx * op.L)
    nres = np.empty(eps.size)
    gres = np.zeros(1)
    neps = np.zeros(1)
    check(lib().fhs_update_dual_data_fidelity(op.handle, dptr(v2f), dptr(yf), dptr(xc.reshape(-1, order="F")),
                                              dptr(Fo_flat), dptr(eps), dptr(s22), dptr(Ftx), dptr(nres),
                                              dptr(gres), dptr(neps)))
    v2c = v2f.view(np.complex128)
    v2_out, nr_out, pos, bpos = [], [], 0, 0
    for l in range(op.L):
        v2_out.append(op.split(l, v2c[pos:pos + op.n_vis[l]]))
        nb = len(op.block_sizes[l])
        nr_out.append(list(nres[bpos:bpos + nb]))
        pos += op.n_vis[l]
        bpos += nb
    Fx_new = Fo_flat.view(np.complex128).reshape(op.L, op.No).T.copy(order="F")
    return (v2_out, Ftx.reshape(op.Ny, op.Nx, op.L, order="F"), Fx_new, nr_out, float(gres[0]),
            float(neps[0]))


def update_dual_data_fidelity_precond(v2, y, x, Fx_old, proj, op: MeasurementOperator, epsilon,
                                      elipse_proj_max_iter, elipse_proj_min_iter, elipse_proj_eps, sigma22):
    """src/update_dual_data_fidelity.m:1-6, 126-147 (no DR) with the
    operator's preconditioner (``op.set_preconditioner``).

    Returns (v2, Ftx, Fx_old, proj, norm_res, global_norm_res, norm_epsilon,
    fb_iters), the reference's outputs plus the FB iterations per block."""
    xc = _cube_in(x, op.Ny, op.Nx)
    v2f = _cplx_in(np.concatenate([op.flatten(v) for v in v2])).copy()
    pjf = _cplx_in(np.concatenate([op.flatten(v) for v in proj])).copy()
    yf = _cplx_in(np.concatenate([op.flatten(v) for v in y]))
    Fo = np.asfortranarray(np.asarray(Fx_old, dtype=np.complex128).reshape(op.No, op.L, order="F"))
    Fo_flat = np.ascontiguousarray(Fo.T).view(np.float64).copy()
    eps = np.concatenate([np.asarray(e, dtype=np.float64).ravel() for e in epsilon])
    s22 = _f64(np.broadcast_to(np.asarray(sigma22, dtype=np.float64), (op.L,)))
    Ftx = np.empty(op.Ny * op.Nx * op.L)
    nres = np.empty(eps.size)
    gres = np.zeros(1)
    neps = np.zeros(1)
    its = np.zeros(eps.size, dtype=np.int32)
    check(lib().fhs_update_dual_data_fidelity_precond(
        op.handle, dptr(v2f), dptr(pjf), dptr(yf), dptr(xc.reshape(-1, order="F")), dptr(Fo_flat), dptr(eps),
        int(elipse_proj_max_iter), int(elipse_proj_min_iter), float(elipse_proj_eps), dptr(s22), dptr(Ftx),
        dptr(nres), dptr(gres), dptr(neps), its.ctypes.data_as(C.POINTER(C.c_int))))
    v2c, pjc = v2f.view(np.complex128), pjf.view(np.complex128)
    v2_out, pj_out, nr_out, it_out, pos, bpos = [], [], [], [], 0, 0
    for l in range(op.L):
        v2_out.append(op.split(l, v2c[pos:pos + op.n_vis[l]]))
        pj_out.append(op.split(l, pjc[pos:pos + op.n_vis[l]]))
        nb = len(op.block_sizes[l])
        nr_out.append(list(nres[bpos:bpos + nb]))
        it_out.append([int(v) for v in its[bpos:bpos + nb]])
        pos += op.n_vis[l]
        bpos += nb
    Fx_new = Fo_flat.view(np.complex128).reshape(op.L, op.No).T.copy(order="F")
    return (v2_out, Ftx.reshape(op.Ny, op.Nx, op.L, order="F"), Fx_new, pj_out, nr_out, float(gres[0]),
            float(neps[0]), it_out)


# ------------------------------------------------------------------- solvers
_PARAM_DEFAULTS = dict(
    nu0=1.0, nu1=1.0, reweighting_alpha=1.0, reweighting_flag=True, reweighting_min_iter=1,
    reweighting_max_iter=20, reweighting_rel_var=1e-4, pdfb_min_iter=10, pdfb_max_iter=2000,
    pdfb_rel_var=5e-5, pdfb_fidelity_tolerance=1.01, pdfb_rel_var_low=5e-6,
    elipse_proj_max_iter=20, elipse_proj_min_iter=1, elipse_proj_eps=1e-8,
    adjust_flag_noise=False, adjust_noise_min_iter=100, adjust_noise_rel_var=1e-3,
    adjust_noise_start_iter=2000, adjust_noise_change_percentage=0.5, alph=1.0, alph_bar=1.0)


class Solver:
    """One primal-dual solver on the GPU (facetHyperSARA / hyperSARA / sara).

    ``param``: dict with the reference's ``param`` fields (imaging/imaging.m:839-860):
    nu2 [L], gamma (per group), gamma0 (per group x facet), reweighting_sig,
    reweighting_sig_bar, reweighting_*, pdfb_*, elipse_proj_*.  A solver
    initialised on an operator with a preconditioner runs the ellipsoid
    projection (the reference's default data term), else the l2-ball form.
    """

    def __init__(self, op: MeasurementOperator, algo: int, param: dict, nlevel=4, n_groups=1, Qy=1, Qx=1,
                 overlap=(0, 0), window="triangular", splits_y=None, splits_x=None):
        self.op = op
        self.algo = algo
        cfg = LB.SolverConfig()
        cfg.algo = algo
        cfg.nlevel = nlevel
        cfg.n_groups = n_groups
        cfg.Qy, cfg.Qx = Qy, Qx
        self._sy = None if splits_y is None else (C.c_int * (Qy + 1))(*[int(v) for v in splits_y])
        self._sx = None if splits_x is None else (C.c_int * (Qx + 1))(*[int(v) for v in splits_x])
        cfg.splits_y = C.cast(self._sy, C.POINTER(C.c_int)) if self._sy is not None else None
        cfg.splits_x = C.cast(self._sx, C.POINTER(C.c_int)) if self._sx is not None else None
        cfg.overlap_y, cfg.overlap_x = int(overlap[0]), int(overlap[1])
        cfg.window = LB.WINDOW_TRIANGULAR if window == "triangular" else LB.WINDOW_NONE
        h = C.c_void_p()
        check(lib().fhs_solver_create(op.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self.G = op.L if algo == LB.ALGO_SARA else n_groups
        self.Q = 0 if algo == LB.ALGO_SARA else (Qy * Qx if algo == LB.ALGO_FHS else 1)
        self.set_params(param)

    def set_params(self, param: dict):
        p = dict(_PARAM_DEFAULTS)
        p.update(param)
        self._arrays = {}

        def arr(key, n):
            a = _f64(np.broadcast_to(np.asarray(p[key], dtype=np.float64).ravel(), (n,)) if np.size(p[key]) == 1
                     else np.asarray(p[key], dtype=np.float64).ravel())
            if a.size != n:
                raise ValueError(f"param {key}: expected {n} values, got {a.size}")
            self._arrays[key] = a
            return dptr(a)

        sp = LB.SolverParams()
        sp.nu0, sp.nu1 = float(p["nu0"]), float(p["nu1"])
        sp.nu2 = arr("nu2", self.op.L)
        sp.gamma = arr("gamma", self.G)
        sp.reweighting_sig = arr("reweighting_sig", self.G)
        if self.Q:
            sp.gamma0 = arr("gamma0", self.G * self.Q)
            sp.reweighting_sig_bar = arr("reweighting_sig_bar", self.G * self.Q)
        sp.reweighting_alpha = float(p["reweighting_alpha"])
        sp.reweighting_flag = int(bool(p["reweighting_flag"]))
        sp.reweighting_min_iter = int(p["reweighting_min_iter"])
        sp.reweighting_max_iter = int(p["reweighting_max_iter"])
        sp.reweighting_rel_var = float(p["reweighting_rel_var"])
        sp.pdfb_min_iter = int(p["pdfb_min_iter"])
        sp.pdfb_max_iter = int(p["pdfb_max_iter"])
        sp.pdfb_rel_var = float(p["pdfb_rel_var"])
        sp.pdfb_fidelity_tolerance = float(p["pdfb_fidelity_tolerance"])
        sp.pdfb_rel_var_low = float(p["pdfb_rel_var_low"])
        sp.elipse_proj_max_iter = int(p["elipse_proj_max_iter"])
        sp.elipse_proj_min_iter = int(p["elipse_proj_min_iter"])
        sp.elipse_proj_eps = float(p["elipse_proj_eps"])
        sp.adjust_flag_noise = int(bool(p["adjust_flag_noise"]))
        sp.adjust_noise_min_iter = int(p["adjust_noise_min_iter"])
        sp.adjust_noise_rel_var = float(p["adjust_noise_rel_var"])
        sp.adjust_noise_start_iter = int(p["adjust_noise_start_iter"])
        sp.adjust_noise_change_percentage = float(p["adjust_noise_change_percentage"])
        sp.alph, sp.alph_bar = float(p["alph"]), float(p["alph_bar"])
        check(lib().fhs_solver_set_params(self._h, C.byref(sp)))

    def set_data(self, y, epsilon):
        yf = _cplx_in(np.concatenate([self.op.flatten(v) for v in y]))
        eps = _f64(np.concatenate([np.asarray(e, dtype=np.float64).ravel() for e in epsilon]))
        check(lib().fhs_solver_set_data(self._h, dptr(yf), dptr(eps)))

    def init(self, xinit=None):
        if xinit is None:
            check(lib().fhs_solver_init(self._h, None))
        else:
            xc = _cube_in(xinit, self.op.Ny, self.op.Nx)
            check(lib().fhs_solver_init(self._h, dptr(xc.reshape(-1, order="F"))))

    def init_warm(self, net, chunk=16):
        """Initialise from the learned warm start on the device (dirty cube,
        network, fallback rule; fhs_solver_init_warm).  ``net``: a
        ``warmstart.UNet`` on the solver's device.  Returns the decision record."""
        info = LB.WarmInfo()
        check(lib().fhs_solver_init_warm(self._h, net._h, int(chunk), C.byref(info)))
        return {"used": bool(info.used), "objective_warm": info.objective_warm,
                "objective_cold": info.objective_cold, "seconds": info.seconds}

    def iterate(self, n, record=True):
        info = (LB.IterInfo * max(n, 1))() if record else None
        check(lib().fhs_solver_iterate(self._h, n, info))
        if not record:
            return None
        return [dict(rel_val=i.rel_val, residual=i.residual, epsilon=i.epsilon, nuclear=i.nuclear)
                for i in list(info)[:n]]

    def run(self, max_iter=0):
        ri = LB.RunInfo()
        check(lib().fhs_solver_run(self._h, int(max_iter), C.byref(ri)))
        return dict(n_iter=ri.n_iter, n_reweights=ri.n_reweights, converged=bool(ri.converged),
                    rel_val=ri.rel_val, residual=ri.residual, epsilon=ri.epsilon, seconds=ri.seconds,
                    n_noise_adjustments=ri.n_noise_adjustments)

    def epsilon(self):
        """Current l2 bounds as [l][b] (adapted by the noise adjustment of run())."""
        out = np.empty(sum(len(b) for b in self.op.block_sizes))
        check(lib().fhs_solver_epsilon(self._h, dptr(out)))
        res, pos = [], 0
        for bl in self.op.block_sizes:
            res.append(list(out[pos:pos + len(bl)]))
            pos += len(bl)
        return res

    def regularization(self):
        """Current (gamma[groups], gamma0[groups x facets] or None)."""
        g = np.empty(self.G)
        g0 = np.empty(max(self.G * self.Q, 1))
        check(lib().fhs_solver_regularization(self._h, dptr(g), dptr(g0) if self.Q else None))
        return g, (g0 if self.Q else None)

    def update_weights(self):
        check(lib().fhs_solver_update_weights(self._h))

    def group_stats(self):
        """FP64 sums of the last iteration per spectral group, [groups, 4]:
        sum (x - x_prev)^2, sum x^2, sum ||res_b||^2, sum eps_b^2."""
        out = np.empty(self.G * 4)
        check(lib().fhs_solver_group_stats(self._h, dptr(out)))
        return out.reshape(self.G, 4)

    def get_state(self):
        """The solver state the reference checkpoints (facetHyperSARA.m:1071-1107):
        dict xsol/g [Ny, Nx, L], v0 (flat, per group and facet [P_q, lg]),
        v1 [s, L], v2/proj (nested [l][b] complex), weights0 [lg, Q, groups],
        weights1 [s, groups], epsilon (nested [l][b], the current l2 bounds);
        absent fields are omitted."""
        op = self.op
        out = {"epsilon": self.epsilon()}
        for name, f in LB.FIELDS.items():
            n = int(lib().fhs_solver_field_size(self._h, f))
            if n <= 0:
                continue
            a = np.empty(n)
            check(lib().fhs_solver_get_field(self._h, f, dptr(a)))
            if name in ("xsol", "g"):
                a = a.reshape(op.Ny, op.Nx, op.L, order="F")
            elif name == "v1":
                a = a.reshape(-1, op.L, order="F")
            elif name == "weights1":
                a = a.reshape(-1, self.G, order="F")
            elif name == "weights0":
                a = a.reshape(-1, self.Q, self.G, order="F")
            elif name in ("v2", "proj"):
                c, res, pos = a.view(np.complex128), [], 0
                for l in range(op.L):
                    res.append(op.split(l, c[pos:pos + op.n_vis[l]].copy()))
                    pos += op.n_vis[l]
                a = res
            out[name] = a
        return out

    def set_state(self, state):
        """Restores fields of get_state (after init); unknown keys are ignored."""
        if "epsilon" in state:
            e = _f64(np.concatenate([np.asarray(b, dtype=np.float64).ravel() for b in state["epsilon"]]))
            check(lib().fhs_solver_set_epsilon(self._h, dptr(e)))
        for name, f in LB.FIELDS.items():
            if name not in state:
                continue
            n = int(lib().fhs_solver_field_size(self._h, f))
            if n <= 0:
                continue
            v = state[name]
            if name in ("v2", "proj"):
                a = _cplx_in(np.concatenate([self.op.flatten(b) for b in v]))
            else:
                a = _f64(np.asarray(v, dtype=np.float64).reshape(-1, order="F"))
            if a.size != n:
                raise ValueError(f"state field {name}: expected {n} values, got {a.size}")
            check(lib().fhs_solver_set_field(self._h, f, dptr(a)))

    def ellipse_iterations(self):
        """FB iterations of the ellipsoid projection per block in the last
        iteration (nested [l][b]; zeros without a preconditioner)."""
        n = sum(len(b) for b in self.op.block_sizes)
        out = np.zeros(n, dtype=np.int32)
        check(lib().fhs_solver_ellipse_iterations(self._h, out.ctypes.data_as(C.POINTER(C.c_int))))
        res, pos = [], 0
        for bs in self.op.block_sizes:
            res.append([int(v) for v in out[pos:pos + len(bs)]])
            pos += len(bs)
        return res

    def time_iterations(self, n):
        """Device milliseconds of n graph replays (CUDA events on the solver stream)."""
        ms = np.zeros(1)
        check(lib().fhs_solver_time_iterations(self._h, int(n), dptr(ms)))
        return float(ms[0])

    def profile_stages(self, n):
        """Mean device milliseconds per iteration stage over n iterations."""
        k = int(lib().fhs_solver_stage_count())
        ms = np.zeros(k)
        check(lib().fhs_solver_profile_stages(self._h, int(n), dptr(ms)))
        return {lib().fhs_solver_stage_name(i).decode(): float(ms[i]) for i in range(k)}

    def x(self):
        out = np.empty(self.op.Ny * self.op.Nx * self.op.L)
        check(lib().fhs_solver_get_x(self._h, dptr(out)))
        return out.reshape(self.op.Ny, self.op.Nx, self.op.L, order="F")

    def close(self):
        if getattr(self, "_h", None):
            lib().fhs_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def facetHyperSARA(y, epsilon, op: MeasurementOperator, param: dict, Qx, Qy, nlevel=4,
                   window_type="triangular", overlap_size=(0, 0), xinit=None, n_groups=1, splits_y=None,
                   splits_x=None, max_iter=0):
    """src/fhs/facetHyperSARA.m:1-6 -> (xsol [Ny, Nx, L], info).  The
    reference's A, At, G, W are the operator handle and pU its preconditioner
    (none: pU = 1); a DR operator (MeasurementOperator.dimensionality_reduction)
    runs the reference's flag_dimensionality_reduction path."""
    s = Solver(op, LB.ALGO_FHS, param, nlevel, n_groups, Qy, Qx, overlap_size, window_type, splits_y, splits_x)
    try:
        s.set_data(y, epsilon)
        s.init(xinit)
        info = s.run(max_iter)
        return s.x(), info
    finally:
        s.close()


def hyperSARA(y, epsilon, op: MeasurementOperator, param: dict, nlevel=4, xinit=None, n_groups=1, max_iter=0):
    """src/hs/hyperSARA.m:1-3 -> (xsol, info)."""
    s = Solver(op, LB.ALGO_HS, param, nlevel, n_groups)
    try:
        s.set_data(y, epsilon)
        s.init(xinit)
        info = s.run(max_iter)
        return s.x(), info
    finally:
        s.close()


def sara(y, epsilon, op: MeasurementOperator, param: dict, nlevel=4, xinit=None, max_iter=0):
    """src/sara/sara.m:1-3 -> (xsol, info); every channel is its own problem."""
    s = Solver(op, LB.ALGO_SARA, param, nlevel)
    try:
        s.set_data(y, epsilon)
        s.init(xinit)
        info = s.run(max_iter)
        return s.x(), info
    finally:
        s.close()
