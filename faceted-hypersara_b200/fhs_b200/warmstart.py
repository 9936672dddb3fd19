"""Learned warm start of the primal-dual solvers.

A BF16 U-Net (4 levels, 32 base channels, 2,140,065 parameters; kernels in
``csrc/unet.cu``, ABI ``fhs_unet_*``) maps each channel of the normalised
dirty cube -- the back-projection ``real(At(G' y))`` divided by the PSF peak,
``compute_residual_images`` of x = 0 (src/compute_residual_images.m:83-102)
-- to an initial estimate x0.  The solver then runs unchanged from x0 (the
``xinit`` / ``varargin{1}`` of src/fhs/facetHyperSARA.m:1-6, used at
:347-350) to the same stopping rule, so the primal-dual iteration keeps the
last word on the result.  ``warm_start`` falls back to the cold start
(x0 = 0) when the warm start's initial objective is not better:

    F(x) = sum_b max(0, ||y_b - Phi_b x|| - eps_b)
           + sum_g gamma_g ||Psi^T x_g||_{2,1} + sum_g gamma0_g ||x_g||_*

(the l2-ball violation of the data term with unit weight, plus the SARA and
nuclear priors of every spectral sub-cube with the solver's regularisation;
the nuclear term is taken over each whole sub-cube).  At x = 0 only the data
term remains.

Training data are pairs (dirty image, plain-solver solution) per channel,
from seeded synthetic cubes solved by the library's own plain solver
(``training_pairs``); ``train`` runs Adam steps of the library's hand-written
forward and backward kernels.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib as LB
from ._lib import check, lib

N_BASE = 32


def layer_specs(b=N_BASE):
    """(Cin, Cout) of the 3x3 layers in the library's parameter order."""
    return [(1, b), (b, b), (b, 2 * b), (2 * b, 2 * b), (2 * b, 4 * b), (4 * b, 4 * b), (4 * b, 8 * b),
            (8 * b, 8 * b), (8 * b, 4 * b), (8 * b, 4 * b), (4 * b, 4 * b), (4 * b, 2 * b), (4 * b, 2 * b),
            (2 * b, 2 * b), (2 * b, b), (2 * b, b), (b, b)]


def init_params(seed=0, b=N_BASE):
    """He-normal 3x3 weights, zero biases, a small head (outputs start near 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in layer_specs(b):
        out.append(rng.standard_normal(co * ci * 9) * np.sqrt(2.0 / (ci * 9)))
        out.append(np.zeros(co))
    out.append(rng.standard_normal(b) * 1e-2)
    out.append(np.zeros(1))
    return np.concatenate(out).astype(np.float32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class UNet:
    """The warm-start network on one GPU (``fhs_unet_*``)."""

    def __init__(self, device=0, params=None, seed=0):
        h = C.c_void_p()
        check(lib().fhs_unet_create(device, N_BASE, C.byref(h)))
        self._h = h
        self.n_params = int(lib().fhs_unet_n_params(h))
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if getattr(self, "_h", None):
            lib().fhs_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = _f32(p)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        check(lib().fhs_unet_set_params(self._h, _fptr(p)))

    def params(self):
        out = np.empty(self.n_params, np.float32)
        check(lib().fhs_unet_get_params(self._h, _fptr(out)))
        return out

    def forward(self, images):
        """images [n, H, W] -> outputs [n, H, W] (float32)."""
        im = _f32(images)
        n, H, W = im.shape
        out = np.empty_like(im)
        check(lib().fhs_unet_forward(self._h, n, H, W, _fptr(im), _fptr(out)))
        return out

    def gradient(self, images, targets):
        im, tg = _f32(images), _f32(targets)
        n, H, W = im.shape
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        check(lib().fhs_unet_gradient(self._h, n, H, W, _fptr(im), _fptr(tg), _fptr(g), C.byref(loss)))
        return float(loss.value), g

    def train_step(self, images, targets, lr):
        im, tg = _f32(images), _f32(targets)
        n, H, W = im.shape
        loss = C.c_double()
        check(lib().fhs_unet_train_step(self._h, n, H, W, _fptr(im), _fptr(tg), float(lr), C.byref(loss)))
        return float(loss.value)


def train(net: UNet, inputs, targets, steps=500, batch=8, lr=1e-3, seed=0, lr_end=None, log=None):
    """Adam steps on random mini-batches of (input, target) images
    [n, H, W]; the learning rate decays geometrically to lr_end (default
    lr / 10).  Returns the per-step losses."""
    rng = np.random.default_rng(seed)
    n = inputs.shape[0]
    lr_end = lr / 10 if lr_end is None else lr_end
    losses = []
    for k in range(steps):
        idx = rng.choice(n, size=min(batch, n), replace=False)
        # random flips / transposes: the imaging problem has no preferred orientation
        a, b = inputs[idx], targets[idx]
        if rng.random() < 0.5:
            a, b = a[:, ::-1], b[:, ::-1]
        if rng.random() < 0.5:
            a, b = a[:, :, ::-1], b[:, :, ::-1]
        rate = lr * (lr_end / lr) ** (k / max(steps - 1, 1))
        losses.append(net.train_step(np.ascontiguousarray(a), np.ascontiguousarray(b), rate))
        if log and (k % 100 == 0 or k == steps - 1):
            log(f"step {k}: loss {losses[-1]:.4e}")
    return np.array(losses)


def dirty_cube(op, y):
    """Normalised dirty cube [Ny, Nx, L]: real(At(G' y)) / PSF peak per channel
    (src/compute_residual_images.m:83-102 at x = 0)."""
    from .api import compute_residual_images
    return compute_residual_images(np.zeros((op.Ny, op.Nx, op.L)), y, op)


def network_cube(net: UNet, cube, chunk=16):
    """Apply the network to every channel of a cube [Ny, Nx, L] (images are
    [Nx, Ny] in the network's row-major convention), clipped at 0 as the
    primal update of the solvers does (fhs_update_primal.m:33-38)."""
    Ny, Nx, L = cube.shape
    imgs = np.ascontiguousarray(np.moveaxis(cube, 2, 0).transpose(0, 2, 1))   # [L, Nx, Ny]
    out = np.empty_like(imgs, dtype=np.float32)
    for c0 in range(0, L, chunk):
        out[c0:c0 + chunk] = net.forward(imgs[c0:c0 + chunk])
    return np.maximum(np.moveaxis(out.transpose(0, 2, 1), 0, 2), 0.0).astype(np.float64)


def objective(x, op, y, eps, gamma, gamma0, n_groups, nlevel=4):
    """F(x) of the fallback rule (module docstring); x [Ny, Nx, L]."""
    from .api import HS_forward_operator_G, compute_sara_prior, nuclear_norm
    f = 0.0
    if not np.any(x):   # Phi 0 = 0: only the data term, from y alone
        for l in range(op.L):
            for b, yb in enumerate(y[l]):
                f += max(0.0, float(np.linalg.norm(np.asarray(yb))) - float(eps[l][b]))
        return f
    Phix = HS_forward_operator_G(x, op)
    for l in range(op.L):
        for b, (pb, yb) in enumerate(zip(Phix[l], y[l])):
            f += max(0.0, float(np.linalg.norm(np.asarray(yb) - pb)) - float(eps[l][b]))
    lg = op.L // n_groups
    g0 = np.ravel(gamma0)
    Q = max(g0.size // n_groups, 1)   # gamma0 is group-major [g * Q + q]: the group's first facet weight
    for g in range(n_groups):
        xg = x[:, :, g * lg:(g + 1) * lg]
        f += float(np.ravel(gamma)[g]) * compute_sara_prior(xg, nlevel)
        f += float(g0[g * Q]) * nuclear_norm(xg.reshape(-1, lg, order="F"))
    return f


def warm_start_device(net: UNet, solver, chunk=16):
    """The same warm start and fallback rule with every cube kept on the
    GPU (``fhs_solver_init_warm``): the solver (data and parameters set) is
    initialised from the network's estimate or from zero; returns the
    decision record."""
    return solver.init_warm(net, chunk)


def warm_start(net: UNet, op, y, eps, gamma, gamma0, n_groups=1, nlevel=4):
    """x0 for the solver and the decision record: the network's estimate if
    its objective F is below F(0), else zeros (cold start)."""
    t0 = time.perf_counter()
    x0 = network_cube(net, dirty_cube(op, y))
    t_net = time.perf_counter() - t0
    f_warm = objective(x0, op, y, eps, gamma, gamma0, n_groups, nlevel)
    f_cold = objective(np.zeros_like(x0), op, y, eps, gamma, gamma0, n_groups, nlevel)
    use = bool(np.isfinite(f_warm) and f_warm < f_cold)
    return (x0 if use else np.zeros_like(x0)), {"used": use, "objective_warm": f_warm, "objective_cold": f_cold,
                                                 "seconds": time.perf_counter() - t0, "network_seconds": t_net}


def training_pairs(n_cubes, Ny, Nx, L, seed=0, device=0, pdfb_max_iter=150, reweighting_max_iter=1,
                   vis_fraction=0.5, snr_db=40.0):
    """(dirty images, plain-solver solutions), [n_cubes * L, Nx, Ny] each:
    seeded cubes with the hyperSARA generator (power-law cube, Gaussian uv
    coverage scaled per channel, M_l = vis_fraction * N, whitened noise),
    solved by the library's plain HyperSARA solver from x = 0 with the
    stopping rule and the stated schedule."""
    from . import heuristics, synth
    from .api import HS_forward_operator_G, MeasurementOperator, Solver
    ins, outs = [], []
    N = Ny * Nx
    for k in range(n_cubes):
        s = seed + 7919 * k
        rng = np.random.default_rng(s)
        x = synth.sky_cube(Ny, Nx, L, s)
        M = int(vis_fraction * N)
        oy0, ox0 = synth.base_coverage(M, s)
        nu = synth.frequencies(L)
        om = [synth.channel_coverage(oy0, ox0, nu[l], nu[-1]) for l in range(L)]
        bsz = [[M] for _ in range(L)]
        op0 = MeasurementOperator(Ny, Nx, om, bsz, device=device)
        y0 = HS_forward_operator_G(np.moveaxis(x, 0, 2), op0)
        op0.close()
        sig = [synth.noise_sigma(y0[l][0], snr_db) for l in range(L)]
        y = [[(y0[l][0] + sig[l] * synth.noise(M, rng)) / sig[l]] for l in range(L)]
        op = MeasurementOperator(Ny, Nx, om, bsz, [np.full(M, 1.0 / sg) for sg in sig], device=device)
        eps = [synth.l2_bounds(b) for b in bsz]
        nu2 = op.operator_norm(50, 1e-6)
        gam, gam0, *_ = heuristics.compute_noise_level(Ny, Nx, L, np.ones(L), "hs", nu2)
        param = dict(nu2=nu2, gamma=gam, gamma0=gam0, reweighting_sig=gam, reweighting_sig_bar=gam0,
                     pdfb_max_iter=pdfb_max_iter, reweighting_max_iter=reweighting_max_iter)
        sv = Solver(op, LB.ALGO_HS, param, nlevel=4)
        sv.set_data(y, eps)
        sv.init()
        sv.run()
        xs = sv.x()
        sv.close()
        d = dirty_cube(op, y)
        op.close()
        ins.append(np.moveaxis(d, 2, 0).transpose(0, 2, 1))
        outs.append(np.moveaxis(xs, 2, 0).transpose(0, 2, 1))
    return (np.ascontiguousarray(np.concatenate(ins), dtype=np.float32),
            np.ascontiguousarray(np.concatenate(outs), dtype=np.float32))
