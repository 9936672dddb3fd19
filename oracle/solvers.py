"""FP64 CPU restatement of the SARA / HyperSARA / Faceted HyperSARA iterations.

TEST INFRASTRUCTURE ONLY (see ``oracle/nufft.py``).

Arrays are channel-first here: an image cube is ``x[L, Ny, Nx]``.  Each
function cites the reference file it restates.  The data-fidelity dual takes
either the l2-ball form (``pU = 1``, ``update_dual_data_fidelity.m:83``) or,
with a ``Precond``, the preconditioned ellipsoid projection
(``update_dual_data_fidelity.m:126-147``).  Visibility gridding (DR) runs
through the same routines on the DR data term of ``oracle/dr.py``.

The ellipsoid projection ``solver_proj_elipse_fb`` and the uniform-weight
preconditioner ``util_gen_preconditioning_matrix`` belong to the
RI-measurement-operator submodule, which the reference tree does not vendor;
both are restated from the published method (Onose et al. 2017) and pinned by
their optimality conditions and the ``pU = 1`` reduction only (parity of
those two functions against the reference is unpinned).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.special import gammaln

from . import wavelets as wv
from ._par import pmap
from .facets import FacetGeometry
from .nufft import NufftOperator

MATLAB_EPS = np.finfo(np.float64).eps


def _adj(G, v):
    """G' v without copying G: conj(G^T conj(v)) (bit-identical to
    G.conj().T @ v: conjugation is exact and the sums run in the same order)."""
    return np.conj(G.T @ np.conj(v))


# ----------------------------------------------------------------- small ops
def proj_l2ball(x, eps, y):
    """src/proj_l2ball.m:20-22."""
    p = x - y
    nrm = np.linalg.norm(p.ravel())
    return p * min(eps / nrm, 1.0) + y if nrm > 0 else x.copy()


def nuclear_norm(x):
    """src/nuclear_norm.m:25-26 (x [L, Ny, Nx])."""
    L = x.shape[0]
    return float(np.sum(np.linalg.svd(x.reshape(L, -1).T, compute_uv=False)))


def compute_sara_prior(x, nlevel=4):
    """src/compute_sara_prior.m:35-41: sum_i ||(Psit x)_i||_2 over channels."""
    r = wv.sara_analysis(x, nlevel)
    return float(np.sum(np.sqrt(np.sum(r * r, axis=0))))


def primal_update(x, g):
    """src/fhs/fhs_update_primal.m:33-38."""
    xn = np.maximum(x - g, 0.0)
    xhat = 2.0 * xn - x
    return xn, xhat, float(np.sum((x - xn) ** 2)), float(np.sum(xn ** 2))


# -------------------------------------------------------------- data fidelity
@dataclass
class DataTerm:
    """Per-channel measurement blocks: G[l][b] (csr, whitening folded in), y, eps."""
    op: NufftOperator
    G: list
    y: list
    eps: list

    @property
    def L(self):
        return len(self.G)


def forward_operator(x, data: DataTerm, pU=None):
    """lib/operators/HS_forward_operator_G.m:36-52 (no DR); with pU,
    HS_forward_operator_precond_G.m:40-55: sqrt(pU) .* (G A x)."""
    def one(l):
        Fx = data.op.A(x[l])
        if pU is None:
            return [G @ Fx for G in data.G[l]]
        return [np.sqrt(pu) * (G @ Fx) for G, pu in zip(data.G[l], pU[l])]
    return pmap(one, range(data.L))


def adjoint_operator(yb, data: DataTerm, pU=None):
    """lib/operators/HS_adjoint_operator_G.m:42-57 (no DR), real part kept;
    with pU, HS_adjoint_operator_precond_G.m: At(G' (sqrt(pU) .* y))."""
    op = data.op

    def one(l):
        g2 = np.zeros(op.No, dtype=np.complex128)
        for b, (G, v) in enumerate(zip(data.G[l], yb[l])):
            g2 += _adj(G, v if pU is None else np.sqrt(pU[l][b]) * v)
        return np.real(op.At(g2))
    return np.stack(pmap(one, range(data.L))).reshape(data.L, op.Ny, op.Nx)


def uniform_weight_preconditioner(om_y, om_x, Ky, Kx):
    """Uniform-weighting preconditioner (util_gen_preconditioning_matrix of the
    missing submodule, gen_uniform_weight_matrix = true, one sub-pixel, as set
    in imaging/default_parameters.json "preconditioning"): pU = 1 / (number
    of visibilities falling in the same cell of the Ky x Kx Fourier grid),
    cells centred on the grid points."""
    ky = np.mod(np.floor(np.asarray(om_y) * Ky / (2 * np.pi) + 0.5), Ky).astype(np.int64)
    kx = np.mod(np.floor(np.asarray(om_x) * Kx / (2 * np.pi) + 0.5), Kx).astype(np.int64)
    cell = ky + Ky * kx
    cnt = np.bincount(cell, minlength=Ky * Kx)
    return 1.0 / cnt[cell]


def proj_ellipse_fb(s, y, pU, eps, z0, max_itr=20, min_itr=1, stop=1e-8):
    """Projection onto {||z - y|| <= eps} in the metric diag(1/pU):
    argmin_z (z-s)^H diag(1/pU) (z-s)/2 with ||z - y|| <= eps, by
    forward-backward iterations z <- P_B(z - mu (z - s)/pU), mu = min(pU)
    (Onose et al. 2017; solver_proj_elipse_fb of the missing submodule,
    called at src/update_dual_data_fidelity.m:133-135 and src/sara/sara.m:594).
    With pU = 1 one iteration is the exact l2-ball projection of s."""
    mu = float(np.min(pU))
    z = np.array(z0, dtype=np.complex128)
    k = 0
    for k in range(1, max_itr + 1):
        t = z - mu * (z - s) / pU
        zn = proj_l2ball(t, eps, y)
        dz = np.linalg.norm(zn - z)
        nz = np.linalg.norm(zn)
        z = zn
        if k >= min_itr and dz <= stop * nz:
            break
    return z, k


def update_dual_data_fidelity_precond(v2, proj, x, Fx_old, data: DataTerm, pU, sigma22, max_itr=20, min_itr=1,
                                      stop=1e-8):
    """src/update_dual_data_fidelity.m:126-147 with a preconditioner pU[l][b]:
    proj = solver_proj_elipse_fb(v2/pU, r2, y, pU, eps, proj, ...),
    v2 = v2 + pU (r2 - proj).  Returns (v2, proj, Ftx, Fx_old, norm_res,
    global_norm_res^2, norm_epsilon^2)."""
    op = data.op
    Ftx = np.zeros_like(x)
    Fx_new = np.empty_like(Fx_old)

    def one(l):
        Fx = op.A(x[l])
        g2 = np.zeros(op.No, dtype=np.complex128)
        nr, vl, pl = [], [], []
        for b, G in enumerate(data.G[l]):
            r2 = G @ (2.0 * Fx - Fx_old[l])
            s = v2[l][b] / pU[l][b] + r2
            p, _ = proj_ellipse_fb(s, data.y[l][b], pU[l][b], data.eps[l][b], proj[l][b], max_itr, min_itr, stop)
            vb = v2[l][b] + pU[l][b] * (r2 - p)
            vl.append(vb)
            pl.append(p)
            g2 += _adj(G, vb)
            nr.append(np.linalg.norm(G @ Fx - data.y[l][b]))
        return Fx, vl, pl, nr, sigma22[l] * np.real(op.At(g2))

    outs = pmap(one, range(data.L))
    norm_res, v2n, pn = [], [], []
    gres, geps = 0.0, 0.0
    for l, (Fx, vl, pl, nr, ftx) in enumerate(outs):   # channel and block order
        for b, res in enumerate(nr):
            gres += res ** 2
            geps += data.eps[l][b] ** 2
        v2n.append(vl)
        pn.append(pl)
        norm_res.append(nr)
        Fx_new[l] = Fx
        Ftx[l] = ftx
    return v2n, pn, Ftx, Fx_new, norm_res, gres, geps


def update_dual_data_fidelity(v2, x, Fx_old, data: DataTerm, sigma22):
    """src/update_dual_data_fidelity.m:116-147 with pU = 1.

    Returns (v2, Ftx, Fx_old, norm_res, global_norm_res^2, norm_epsilon^2).
    """
    op = data.op
    Ftx = np.zeros_like(x)
    Fx_new = np.empty_like(Fx_old)

    def one(l):
        Fx = op.A(x[l])
        g2 = np.zeros(op.No, dtype=np.complex128)
        nr, vl = [], []
        for b, G in enumerate(data.G[l]):
            r2 = G @ (2.0 * Fx - Fx_old[l])
            p = proj_l2ball(v2[l][b] + r2, data.eps[l][b], data.y[l][b])
            vb = v2[l][b] + r2 - p
            vl.append(vb)
            g2 += _adj(G, vb)
            nr.append(np.linalg.norm(G @ Fx - data.y[l][b]))
        return Fx, vl, nr, sigma22[l] * np.real(op.At(g2))

    outs = pmap(one, range(data.L))
    norm_res, v2n = [], []
    gres, geps = 0.0, 0.0
    for l, (Fx, vl, nr, ftx) in enumerate(outs):   # channel and block order
        for b, res in enumerate(nr):
            gres += res ** 2
            geps += data.eps[l][b] ** 2
        v2n.append(vl)
        norm_res.append(nr)
        Fx_new[l] = Fx
        Ftx[l] = ftx
    return v2n, Ftx, Fx_new, norm_res, gres, geps


def compute_residual_images(x, data: DataTerm):
    """src/compute_residual_images.m:83-102 (no DR): real(At(G'(y - G A x)))
    per channel, normalised by the peak of the PSF real(At(G'G A dirac)),
    dirac at pixel (N/2+1, N/2+1) (1-based)."""
    op = data.op
    out = np.zeros_like(x)
    dirac = np.zeros((op.Ny, op.Nx))
    dirac[op.Ny // 2, op.Nx // 2] = 1.0

    def one(l):
        Fx = op.A(x[l])
        r = np.zeros(op.No, dtype=np.complex128)
        for G, yb in zip(data.G[l], data.y[l]):
            r += _adj(G, yb - G @ Fx)
        res = np.real(op.At(r))
        Fd = op.A(dirac)
        rp = np.zeros(op.No, dtype=np.complex128)
        for G in data.G[l]:
            rp += _adj(G, G @ Fd)
        return res / np.max(np.real(op.At(rp)))
    for l, r in enumerate(pmap(one, range(data.L))):
        out[l] = r
    return out


def operator_norm(data: DataTerm, n_iter=200, tol=1e-8, seed=0, pU=None):
    """Squared spectral norm of Phi_l = G_l A per channel by power iteration
    (lib/utils/util_operator_norm.m:43-61, op_norm of the missing submodule);
    with pU, of sqrt(pU) G_l A (util_operator_norm.m:46-52)."""
    rng = np.random.default_rng(seed)
    op = data.op
    starts = [rng.standard_normal((op.Ny, op.Nx)) for _ in range(data.L)]   # drawn in channel order

    def one(l):
        x = starts[l] / np.linalg.norm(starts[l])
        val = 0.0
        for _ in range(n_iter):
            Fx = op.A(x)
            g2 = np.zeros(op.No, dtype=np.complex128)
            for b, G in enumerate(data.G[l]):
                g2 += _adj(G, G @ Fx if pU is None else pU[l][b] * (G @ Fx))
            xn = np.real(op.At(g2))
            new = np.linalg.norm(xn)
            x = xn / new
            if abs(new - val) <= tol * new:
                val = new
                break
            val = new
        return val
    return np.array(pmap(one, range(data.L)), dtype=np.float64)


# ---------------------------------------------------------------- the priors
def l21_prox_update(v1, xhat, weights1, beta1, nlevel=4):
    """src/hs/hs_update_dual_sparsity_distributed.m:41-54 (and the faceted
    src/fhs/fhs_update_dual_sparsity.m:67-93, whose facet coefficients are the
    global ones).  Returns (v1, Psi v1) (no step size applied)."""
    r1 = v1 + wv.sara_analysis(xhat, nlevel)
    l2 = np.sqrt(np.sum(r1 * r1, axis=0))
    l2_soft = np.maximum(l2 - beta1 * weights1, 0.0) / (l2 + MATLAB_EPS)
    v1 = r1 - l2_soft[None, :] * r1
    n0, n1 = xhat.shape[1:]
    return v1, wv.sara_synthesis(v1, n0, n1, nlevel)


def nuclear_prox_update(v0, xhat_facet, window, weights0, beta0):
    """src/fhs/fhs_update_dual_lowrankness.m:40-45 (window = 1 gives
    src/hs/hs_update_dual_lowrankness_serial.m:37-42 without sigma0).
    v0 [P, L]; xhat_facet [L, ny, nx]; returns (v0, g0 [L, ny, nx])."""
    L, ny, nx = xhat_facet.shape
    Z = v0 + (window[None] * xhat_facet).reshape(L, -1).T
    U, S, Vt = np.linalg.svd(Z, full_matrices=False)
    v0 = Z - (U * np.maximum(S - beta0 * weights0, 0.0)) @ Vt
    g0 = window[None] * v0.T.reshape(L, ny, nx)
    return v0, g0


def nuclear_weights(x_facet_weighted, sig_bar, alpha):
    """src/fhs/fhs_update_weights.m:73-77: weights0 = u/(u + sigma_i)."""
    L = x_facet_weighted.shape[0]
    s = np.linalg.svd(x_facet_weighted.reshape(L, -1).T, compute_uv=False)
    u = sig_bar * alpha
    return u / (u + np.abs(s))


def l21_weights(x, sig, alpha, nlevel=4):
    """src/fhs/fhs_update_weights.m:79-92 (global coefficients)."""
    z = wv.sara_analysis(x, nlevel)
    d = np.sqrt(np.sum(z * z, axis=0))
    u = sig * alpha
    return u / (u + d)


def compute_noise_level(Ny, Nx, L, std_noise, algo, geometry: FacetGeometry | None,
                        squared_operator_norm):
    """src/heuristics/compute_noise_level.m:49-89."""
    std_noise = np.asarray(std_noise, dtype=np.float64)
    son = np.asarray(squared_operator_norm, dtype=np.float64)
    sig_sara = np.sqrt(np.mean(std_noise ** 2 / son))
    mu_chi = np.sqrt(2.0) * np.exp(gammaln((L + 1) / 2.0) - gammaln(L / 2.0))
    sig_chi = np.sqrt(L - mu_chi ** 2)
    sig = sig_sara * (mu_chi + sig_chi)
    s = np.sum(std_noise ** 2 / son)
    if algo == "hs" or geometry is None:
        sig_bar = np.sqrt(Nx * Ny * s / min(Nx * Ny, L))
    else:
        sig_bar = np.array([np.sqrt(geometry.n_pixels(q) * s / min(geometry.n_pixels(q), L))
                            for q in range(geometry.Q)])
    return sig, sig_bar, mu_chi, sig_chi, sig_sara


# ----------------------------------------------------------------- solvers
@dataclass
class SolverParams:
    """The ``param`` struct fields the solvers read (imaging/imaging.m:839-860,
    imaging/default_parameters.json)."""
    nu0: float = 1.0
    nu1: float = 1.0
    nu2: np.ndarray = None
    gamma: float = 1e-3          # mu (l21 / l1)
    gamma0: np.ndarray = None    # mu_bar per facet (or scalar for hs)
    reweighting_sig: float = 1.0
    reweighting_sig_bar: np.ndarray = None
    reweighting_alpha: float = 1.0
    reweighting_flag: bool = True
    reweighting_min_iter: int = 1
    reweighting_max_iter: int = 20
    reweighting_rel_var: float = 1e-4
    pdfb_min_iter: int = 10
    pdfb_max_iter: int = 2000
    pdfb_rel_var: float = 5e-5
    pdfb_fidelity_tolerance: float = 1.01
    pdfb_rel_var_low: float = 5e-6
    nlevel: int = 4
    # noise-level adjustment (facetHyperSARA.m:503-526, 877-951)
    adjust_flag_noise: bool = False
    adjust_noise_min_iter: int = 100
    adjust_noise_rel_var: float = 1e-3
    adjust_noise_start_iter: int = 2000
    adjust_noise_change_percentage: float = 0.5
    alph: float = 1.0
    alph_bar: float = 1.0


@dataclass
class SolverLog:
    rel_val: list = field(default_factory=list)
    residual: list = field(default_factory=list)
    epsilon: list = field(default_factory=list)
    n_iter: int = 0
    n_reweights: int = 0


def _stop_pdfb(t, last, rel, res, epsn, p: SolverParams):
    """src/fhs/facetHyperSARA.m:877-881."""
    return (t - last >= p.pdfb_min_iter) and (
        t - last >= p.pdfb_max_iter
        or (rel <= p.pdfb_rel_var and res <= p.pdfb_fidelity_tolerance * epsn)
        or rel <= p.pdfb_rel_var_low)


@dataclass
class Precond:
    """Preconditioning matrices pU[l][b] (diagonal, one vector per block) and
    the ``elipse_proj_*`` parameters (imaging/default_parameters.json)."""
    pU: list
    max_itr: int = 20
    min_itr: int = 1
    stop: float = 1e-8


def _dual_step(v2, proj, x, Fx_old, data, sigma22, pc: Precond | None):
    if pc is None:
        v2, Ftx, Fx_old, nres, gres, geps = update_dual_data_fidelity(v2, x, Fx_old, data, sigma22)
        return v2, proj, Ftx, Fx_old, gres, geps, nres
    v2, proj, Ftx, Fx_old, nres, gres, geps = update_dual_data_fidelity_precond(
        v2, proj, x, Fx_old, data, pc.pU, sigma22, pc.max_itr, pc.min_itr, pc.stop)
    return v2, proj, Ftx, Fx_old, gres, geps, nres


def adjust_noise_trigger(algo, t, last, rel, res, epsn, p: SolverParams):
    """pdfb_adjust_noise of facetHyperSARA.m:883-889 ('fhs': also at the
    first iteration of the run) and hyperSARA.m:690-695 ('hs': at
    adjust_noise_start_iter instead)."""
    if not (res > p.pdfb_fidelity_tolerance * epsn):
        return False
    early = last < 1 if algo == "fhs" else (last < 1 and t == p.adjust_noise_start_iter)
    return (t - last >= p.pdfb_max_iter or early
            or (rel <= p.adjust_noise_rel_var and t - last >= p.adjust_noise_min_iter))


def adjust_noise(eps, norm_res, block_sizes, p: SolverParams):
    """facetHyperSARA.m:906-920: eps_b <- (eps_b + ||res_b||) c where
    eps_b < (2 - tol) ||res_b||, then the channel noise level.  The reference
    takes std() of a fresh randn draw with per-block sigma^2 = eps_b^2 / M_b;
    this returns its expectation sqrt(sum_b eps_b^2 / sum_b M_b) (the draw
    scatters around it by ~1/sqrt(2 M)).  Returns (eps, sigma per channel)."""
    out, sig = [], []
    for el, rl, ml in zip(eps, norm_res, block_sizes):
        e = [(eb + rb) * p.adjust_noise_change_percentage
             if eb < (2.0 - p.pdfb_fidelity_tolerance) * rb else eb for eb, rb in zip(el, rl)]
        out.append(e)
        m = float(sum(ml))
        sig.append(float(np.sqrt(sum(v * v for v in e) / m)) if m > 0 else 0.0)
    return out, np.array(sig)


class FhsIteration:
    """State of one Faceted HyperSARA sub-cube between iterations
    (src/fhs/facetHyperSARA.m:701-889): ``step()`` runs one primal-dual
    iteration, ``reweight()`` the weight update of :952-1137.  Initial duals
    and weights as src/fhs/fhs_initialize_dual_and_weights.m:88-118; proj
    starts at zero (src/fhs/fhs_initialize_data_worker.m:43)."""

    def __init__(self, data: DataTerm, p: SolverParams, geom: FacetGeometry, xinit=None,
                 precond: Precond | None = None):
        op = data.op
        L = data.L
        self.data, self.p, self.geom, self.precond = data, p, geom, precond
        self.x = np.zeros((L, op.Ny, op.Nx)) if xinit is None else np.array(xinit, dtype=np.float64)
        tau = 0.99 / 3.0
        self.sigma0, self.sigma1 = 1.0 / p.nu0, 1.0 / p.nu1
        self.sigma00, self.sigma11 = tau * self.sigma0, tau * self.sigma1
        self.sigma22 = tau / np.asarray(p.nu2, dtype=np.float64)
        self.beta0 = np.asarray(p.gamma0, dtype=np.float64) / self.sigma0 * np.ones(geom.Q)
        self.beta1 = p.gamma / self.sigma1
        self.sig_bar = np.asarray(p.reweighting_sig_bar, dtype=np.float64) * np.ones(geom.Q)
        self.facets = list(geom.facets())
        x = self.x
        self.v0, self.w0 = [], []
        zero = np.linalg.norm(x) == 0
        for q, (y0, y1), (x0, x1), win in self.facets:
            self.v0.append(np.zeros(((y1 - y0) * (x1 - x0), L)))
            self.w0.append(np.ones(L) if zero else
                           nuclear_weights(win[None] * x[:, y0:y1, x0:x1], self.sig_bar[q], p.reweighting_alpha))
        s = wv.n_coefs_sara(op.Ny, op.Nx, p.nlevel)
        self.v1 = np.zeros((L, s))
        self.w1 = np.ones(s) if zero else l21_weights(x, p.reweighting_sig, p.reweighting_alpha, p.nlevel)
        self.v2 = [[np.zeros_like(yb) for yb in data.y[l]] for l in range(L)]
        self.proj = [[np.zeros_like(yb) for yb in data.y[l]] for l in range(L)]
        self.Fx_old = np.stack([op.A(x[l]) for l in range(L)])
        self.g = np.zeros_like(x)

    def step(self):
        """One iteration; returns (sum (x - x_prev)^2, sum x^2, sum_b ||res_b||^2,
        sum_b eps_b^2, norm_res per block)."""
        x, xhat, rel_x, norm_x = primal_update(self.x, self.g)
        self.x = x
        self.v2, self.proj, Ftx, self.Fx_old, gres, geps, nres = _dual_step(
            self.v2, self.proj, x, self.Fx_old, self.data, self.sigma22, self.precond)
        gacc = np.zeros_like(x)
        prox = pmap(lambda f: nuclear_prox_update(self.v0[f[0]], xhat[:, f[1][0]:f[1][1], f[2][0]:f[2][1]], f[3],
                                                  self.w0[f[0]], self.beta0[f[0]]), self.facets)
        for (q, (y0, y1), (x0, x1), win), (v0q, g0) in zip(self.facets, prox):   # overlaps summed in facet order
            self.v0[q] = v0q
            gacc[:, y0:y1, x0:x1] += self.sigma00 * g0
        self.v1, g1 = l21_prox_update(self.v1, xhat, self.w1, self.beta1, self.p.nlevel)
        self.g = gacc + self.sigma11 * g1 + Ftx
        return rel_x, norm_x, gres, geps, nres

    def reweight(self):
        """src/fhs/fhs_update_weights.m:73-92 from the current x."""
        x, p = self.x, self.p
        for q, (y0, y1), (x0, x1), win in self.facets:
            self.w0[q] = nuclear_weights(win[None] * x[:, y0:y1, x0:x1], self.sig_bar[q], p.reweighting_alpha)
        self.w1 = l21_weights(x, p.reweighting_sig, p.reweighting_alpha, p.nlevel)


def facet_hypersara(data: DataTerm, p: SolverParams, geom: FacetGeometry,
                    xinit=None, max_iter=None, callback=None, precond: Precond | None = None,
                    algo: str = "fhs"):
    """src/fhs/facetHyperSARA.m:701-1138 (one spectral sub-cube)."""
    op = data.op
    L = data.L
    adjust = bool(p.adjust_flag_noise)
    if adjust:
        # the l2 bounds change: work on a copy
        data = DataTerm(data.op, data.G, data.y, [list(e) for e in data.eps])
    it = FhsIteration(data, p, geom, xinit, precond)
    log = SolverLog()
    x_last_rw = it.x.copy()
    last, rw_count = 0, 0
    max_iter = max_iter or (p.reweighting_max_iter + 1) * p.pdfb_max_iter
    if adjust:
        # priors off from the first iteration until the first adjustment
        # (facetHyperSARA.m:704-708)
        it.beta0, it.beta1 = np.zeros(geom.Q), 0.0
    for t in range(1, max_iter + 1):
        rel_x, norm_x, gres, geps, nres = it.step()
        x = it.x
        rel = np.sqrt(rel_x / norm_x) if norm_x > 0 else 0.0
        res, epsn = np.sqrt(gres), np.sqrt(geps)
        log.rel_val.append(rel)
        log.residual.append(res)
        log.epsilon.append(epsn)
        log.n_iter = t
        if callback is not None:
            callback(t, x)
        if adjust and adjust_noise_trigger(algo, t, last, rel, res, epsn, p):
            # facetHyperSARA.m:903-944 / hyperSARA.m:697-733
            eps_new, sig_ch = adjust_noise(data.eps, nres, [[len(yb) for yb in yl] for yl in data.y], p)
            data.eps[:] = eps_new
            sig_n, sig_bar_n, *_ = compute_noise_level(op.Ny, op.Nx, L, sig_ch, algo,
                                                       geom if algo == "fhs" else None, p.nu2)
            it.beta1 = p.alph * sig_n / it.sigma1
            it.beta0 = p.alph_bar * np.asarray(sig_bar_n, dtype=np.float64) * np.ones(geom.Q) / it.sigma0
            log.n_adjust = getattr(log, "n_adjust", 0) + 1
            last = t
            continue
        if _stop_pdfb(t, last, rel, res, epsn, p):
            adjust = False
            rel_rw = np.linalg.norm(x_last_rw - x) / max(np.linalg.norm(x_last_rw), 1e-300)
            if (not p.reweighting_flag) or (rw_count >= p.reweighting_min_iter and (
                    rw_count >= p.reweighting_max_iter or rel_rw <= p.reweighting_rel_var)):
                break
            it.reweight()
            x_last_rw = x.copy()
            rw_count += 1
            last = t
    log.n_reweights = rw_count
    log.epsilon_final = [list(e) for e in data.eps]
    return it.x, log


def hypersara(data: DataTerm, p: SolverParams, xinit=None, max_iter=None, callback=None,
              precond: Precond | None = None):
    """src/hs/hyperSARA.m:565-866 (no faceting)."""
    op = data.op
    geom = FacetGeometry(op.Ny, op.Nx, 1, 1, (0, 0), window_type="none")
    # HyperSARA is the Q = 1 faceted iteration without window; its g0 scaling
    # (sigma0 inside hs_update_dual_lowrankness_serial.m:42) equals sigma00
    # because hyperSARA.m:476 also builds sigma00 = tau*sigma0.
    return facet_hypersara(data, p, geom, xinit, max_iter, callback, precond, algo="hs")


def sara(data: DataTerm, p: SolverParams, xinit=None, max_iter=None, callback=None,
         precond: Precond | None = None):
    """src/sara/sara.m:521-837 (single channel, per-basis l1 prox).  With a
    preconditioner, proj starts as the projection of G A x0 from zero
    (src/sara/sara.m:420-428)."""
    op = data.op
    assert data.L == 1
    x = np.zeros((1, op.Ny, op.Nx)) if xinit is None else np.array(xinit, dtype=np.float64).reshape(1, op.Ny, op.Nx)
    sigma1 = 1.0 / p.nu1
    sigma2 = 1.0 / float(np.asarray(p.nu2).ravel()[0])
    tau = 0.99 / (sigma1 * p.nu1 + sigma2 * float(np.asarray(p.nu2).ravel()[0]))
    sigma11, sigma22 = tau * sigma1, tau * sigma2
    beta1 = p.gamma / sigma1
    u = p.reweighting_sig * p.reweighting_alpha
    w1 = u / (u + np.abs(wv.sara_analysis(x[0], p.nlevel)))      # sara.m:352-362
    v1 = np.zeros_like(w1)
    v2 = [[np.zeros_like(yb) for yb in data.y[0]]]
    Fx_old = np.stack([op.A(x[0])])
    proj = None
    if precond is not None:
        proj = [[proj_ellipse_fb(G @ Fx_old[0], yb, pu, e, np.zeros_like(yb), precond.max_itr,
                                 precond.min_itr, precond.stop)[0]
                 for G, yb, pu, e in zip(data.G[0], data.y[0], precond.pU[0], data.eps[0])]]
    g = np.zeros_like(x)
    log = SolverLog()
    x_last_rw = x.copy()
    last, rw_count = 0, 0
    max_iter = max_iter or (p.reweighting_max_iter + 1) * p.pdfb_max_iter
    for t in range(1, max_iter + 1):
        x, xhat, rel_x, norm_x = primal_update(x, g)
        r1 = v1 + wv.sara_analysis(xhat[0], p.nlevel)                # run_par_waverec
        v1 = r1 - np.sign(r1) * np.maximum(np.abs(r1) - beta1 * w1, 0.0)
        g1 = wv.sara_synthesis(v1, op.Ny, op.Nx, p.nlevel)
        v2, proj, Ftx, Fx_old, gres, geps, _ = _dual_step(v2, proj, x, Fx_old, data, [1.0], precond)
        g = sigma11 * g1[None] + sigma22 * Ftx                        # sara.m:633
        rel = np.sqrt(rel_x / norm_x) if norm_x > 0 else 0.0
        res, epsn = np.sqrt(gres), np.sqrt(geps)
        log.rel_val.append(rel)
        log.residual.append(res)
        log.epsilon.append(epsn)
        log.n_iter = t
        if callback is not None:
            callback(t, x)
        if _stop_pdfb(t, last, rel, res, epsn, p):
            rel_rw = np.linalg.norm(x_last_rw - x) / max(np.linalg.norm(x_last_rw), 1e-300)
            if (not p.reweighting_flag) or (rw_count >= p.reweighting_min_iter and (
                    rw_count >= p.reweighting_max_iter or rel_rw <= p.reweighting_rel_var)):
                break
            w1 = u / (u + np.abs(wv.sara_analysis(x[0], p.nlevel)))   # sara.m:764-768
            x_last_rw = x.copy()
            rw_count += 1
            last = t
    log.n_reweights = rw_count
    return x[0], log


def snr_db(x_true, x):
    return 20.0 * np.log10(np.linalg.norm(x_true) / np.linalg.norm(x_true - x))
