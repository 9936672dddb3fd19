"""CPU checks of the FP64 oracle: known answers, invariants, golden fixtures.

The reference cannot run here (MATLAB, un-vendored submodules) and ships no
tests, so the oracle is pinned by mathematical known answers (exact NUDFT,
the closed-form db2 filter, orthonormality and vanishing moments, perfect
reconstruction, adjointness, prox identities) and by the committed fixtures
of tests/golden/ (regenerated by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from fhs_b200 import synth
from oracle import nufft, problem, wavelets
from oracle import solvers as so
from oracle.facets import FacetGeometry, split_range

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


# ---------------------------------------------------------------- NUFFT
@pytest.mark.parametrize("N", [16, 32, 40])
def test_nufft_matches_exact_nudft(N):
    rng = np.random.default_rng(N)
    op = nufft.NufftOperator(N, N)
    om = rng.uniform(-np.pi, np.pi, size=(300, 2))
    x = rng.standard_normal((N, N))
    y = op.G(om[:, 0], om[:, 1]) @ op.A(x)
    ye = nufft.nudft(x, om[:, 0], om[:, 1])
    assert np.linalg.norm(y - ye) / np.linalg.norm(ye) < 2e-5


def test_nufft_adjoint_identity():
    rng = np.random.default_rng(1)
    op = nufft.NufftOperator(24, 20)
    om = rng.uniform(-np.pi, np.pi, size=(200, 2))
    G = op.G(om[:, 0], om[:, 1])
    x = rng.standard_normal((24, 20))
    y = rng.standard_normal(200) + 1j * rng.standard_normal(200)
    lhs = np.vdot(y, G @ op.A(x))
    rhs = np.vdot(op.At(G.conj().T @ y), x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_scaling_fit_tracks_kaiser_bessel():
    a = nufft.scaling_cosine_coefs(64, 128, 7)
    s = nufft.scaling_factors(64, 128, 7, a)
    n = np.arange(64)
    kb = nufft.kb_ft(0, 7, 2.34 * 7) / nufft.kb_ft((n - 31.5) / 128, 7, 2.34 * 7)
    assert np.max(np.abs(s - kb) / kb) < 1e-4


def test_nufft_golden():
    g = _load("nufft_16x12.npz")
    op = nufft.NufftOperator(16, 12)
    assert np.allclose(op.A(g["x"]), g["Fx"], rtol=1e-12, atol=1e-12)
    y = op.G(g["om_y"], g["om_x"]) @ op.A(g["x"])
    assert np.allclose(y, g["y"], rtol=1e-12, atol=1e-12)


# ---------------------------------------------------------------- wavelets
def test_db2_closed_form():
    s3 = np.sqrt(3.0)
    ref = np.array([1 + s3, 3 + s3, 3 - s3, 1 - s3]) / (4 * np.sqrt(2))
    assert np.allclose(wavelets.daubechies_lo_r(2), ref, atol=1e-14)


@pytest.mark.parametrize("p", range(1, 9))
def test_daubechies_orthonormal_and_vanishing_moments(p):
    h = wavelets.daubechies_lo_r(p)
    L = len(h)
    assert L == 2 * p
    assert abs(np.sum(h) - np.sqrt(2)) < 1e-12
    for m in range(p):
        assert abs(np.sum(h[: L - 2 * m] * h[2 * m:]) - (1.0 if m == 0 else 0.0)) < 1e-10
    k = np.arange(L)
    for q in range(p):
        assert abs(np.sum((-1.0) ** k * k ** q * h)) < 1e-8 * max(1, L ** q)
    g = _load("daubechies.npz")
    assert np.allclose(h, g[f"db{p}"], atol=1e-13)


@pytest.mark.parametrize("shape", [(13, 10), (32, 32), (7, 40)])
def test_sara_perfect_reconstruction_and_adjoint(shape):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal((2,) + shape)
    c = wavelets.sara_analysis(x)
    assert c.shape[-1] == wavelets.n_coefs_sara(*shape)
    assert np.allclose(wavelets.sara_synthesis(c, *shape), x, atol=1e-10)
    d = rng.standard_normal(c.shape)
    assert abs(np.sum(d * c) - np.sum(wavelets.sara_synthesis(d, *shape) * x)) < 1e-9 * np.abs(d * c).sum()
    assert abs(np.linalg.norm(c) / np.linalg.norm(x) - 1.0) < 1e-10  # Parseval frame


def test_sara_coefficient_counts():
    # s/N for zero padding with db1..db8 + Dirac at 4 levels
    for n, ratio in ((256, 9.9256), (512, 9.4433), (1024, 9.2168)):
        assert abs(wavelets.n_coefs_sara(n, n) / (n * n) - ratio) < 1e-3


def test_sara_golden():
    g = _load("sara_13x10x2.npz")
    assert np.allclose(wavelets.sara_analysis(g["x"]), g["coefs"], atol=1e-12)


# ---------------------------------------------------------------- prox / priors
def test_proj_l2ball_moreau_identity():
    rng = np.random.default_rng(3)
    y = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    for scale in (0.01, 10.0):
        z = y + scale * (rng.standard_normal(50) + 1j * rng.standard_normal(50))
        p = so.proj_l2ball(z, 2.0, y)
        assert np.linalg.norm(p - y) <= 2.0 + 1e-12
        # dual form used by the solvers: v = z - y - P_B(0,eps)(z - y)
        w = z - y
        v = w * (1 - min(2.0 / np.linalg.norm(w), 1))
        assert np.allclose(v, z - p, atol=1e-12)


def test_gram_eig_prox_equals_svd_prox():
    """fhs_update_dual_lowrankness.m:42-44 restated as Z (I - V diag(shrink) V^T)."""
    rng = np.random.default_rng(5)
    Z = rng.standard_normal((300, 6)) @ np.diag([10, 5, 2, 1, 0.5, 0.1])
    w = rng.uniform(0.2, 1.0, 6)
    beta = 1.5
    U, S, Vt = np.linalg.svd(Z, full_matrices=False)
    ref = Z - (U * np.maximum(S - beta * w, 0)) @ Vt
    lam, V = np.linalg.eigh(Z.T @ Z)
    order = np.argsort(lam)[::-1]
    lam, V = lam[order], V[:, order]
    sig = np.sqrt(np.maximum(lam, 0))
    shrink = np.where(sig > 0, np.maximum(sig - beta * w, 0) / np.where(sig > 0, sig, 1), 0)
    out = Z @ (np.eye(6) - (V * shrink) @ V.T)
    assert np.allclose(out, ref, atol=1e-10)


def test_l21_prox_reduces_to_l1_for_one_channel():
    rng = np.random.default_rng(8)
    x = rng.standard_normal((1, 16, 16))
    v1 = np.zeros((1, wavelets.n_coefs_sara(16, 16)))
    w1 = rng.uniform(0.5, 1.0, v1.shape[1])
    v_l21, _ = so.l21_prox_update(v1, x, w1, 0.3)
    r1 = wavelets.sara_analysis(x)
    v_l1 = r1 - np.sign(r1) * np.maximum(np.abs(r1) - 0.3 * w1, 0)
    assert np.allclose(v_l21, v_l1, atol=1e-12)


def test_nuclear_norm_and_sara_prior_values():
    rng = np.random.default_rng(9)
    x = rng.standard_normal((3, 8, 8))
    assert abs(so.nuclear_norm(x) - np.sum(np.linalg.svd(x.reshape(3, -1).T, compute_uv=False))) < 1e-12
    c = wavelets.sara_analysis(x)
    assert abs(so.compute_sara_prior(x) - np.sum(np.sqrt(np.sum(c * c, axis=0)))) < 1e-12


# ---------------------------------------------------------------- facets / heuristics
def test_split_range_and_windows_partition_of_unity():
    assert split_range(4, 10) == [(0, 3), (3, 5), (5, 8), (8, 10)]  # round half away from zero
    assert split_range(3, 12, 2) == [(0, 4), (2, 8), (6, 12)]
    g = FacetGeometry(40, 30, 3, 2, (4, 3), splits_y=[0, 12, 27, 40])
    total = np.zeros((40, 30))
    for q, (y0, y1), (x0, x1), w in g.facets():
        total[y0:y1, x0:x1] += w
    assert np.allclose(total, 1.0)


def test_noise_level_product_matches_oracle():
    from fhs_b200 import heuristics
    nu2 = np.array([100.0, 150.0, 220.0])
    geom = FacetGeometry(64, 48, 2, 3, (5, 4), splits_y=[0, 30, 64], splits_x=[0, 15, 33, 48])
    ref = so.compute_noise_level(64, 48, 3, np.ones(3), "fhs", geom, nu2)
    out = heuristics.compute_noise_level(64, 48, 3, np.ones(3), "fhs", nu2, [0, 30, 64], [0, 15, 33, 48], (5, 4))
    assert np.isclose(out[0], ref[0]) and np.allclose(out[1], ref[1])
    ref_hs = so.compute_noise_level(64, 48, 3, np.ones(3), "hs", None, nu2)
    out_hs = heuristics.compute_noise_level(64, 48, 3, np.ones(3), "hs", nu2)
    assert np.isclose(out_hs[1], ref_hs[1])


def test_synthetic_generators_are_seeded():
    a = synth.sky_image(32, 32, 5)
    assert np.array_equal(a, synth.sky_image(32, 32, 5)) and a.min() >= 0
    oy, ox = synth.base_coverage(1000, 3)
    assert np.all(np.abs(oy) <= np.pi) and np.all(np.abs(ox) <= np.pi)
    sizes = synth.split_blocks(1000, 5, np.random.default_rng(0))
    assert sum(sizes) == 1000 and min(sizes) >= 1
    eps = synth.l2_bounds([400, 600])
    assert np.isclose(np.sum(np.square(eps)), 1000 + 2 * np.sqrt(1000))
    sp = synth.jittered_splits(4, 1024, 0.15, np.random.default_rng(1))
    assert sp[0] == 0 and sp[-1] == 1024 and np.all(np.diff(sp) > 0)


# ---------------------------------------------------------------- solver golden
def test_fhs_iterations_golden():
    g = _load("fhs_24x24x2_3iter.npz")
    data, xt, meta = problem.make_problem(24, 24, 2, 300, 2, seed=7, synth=synth)
    geom = FacetGeometry(24, 24, 2, 2, (3, 3))
    p = so.SolverParams(nu2=g["nu2"], gamma=float(g["sig"]), gamma0=g["sig_bar"], reweighting_sig=float(g["sig"]),
                        reweighting_sig_bar=g["sig_bar"], pdfb_min_iter=10 ** 6, reweighting_flag=False)
    x3, _ = so.facet_hypersara(data, p, geom, max_iter=3)
    assert np.allclose(x3, g["x3"], rtol=1e-10, atol=1e-12)


def test_small_fhs_solve_improves_snr():
    data, xt, meta = problem.make_problem(32, 32, 2, 500, 2, seed=11, synth=synth)
    nu2 = so.operator_norm(data, 100, 1e-8)
    geom = FacetGeometry(32, 32, 2, 2, (4, 4))
    sig, sig_bar, *_ = so.compute_noise_level(32, 32, 2, np.ones(2), "fhs", geom, nu2)
    p = so.SolverParams(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                        pdfb_max_iter=60, reweighting_max_iter=1)
    x, log = so.facet_hypersara(data, p, geom)
    assert so.snr_db(xt, x) > 8.0
    assert log.n_reweights == 1


def test_ellipse_projection_optimality_and_l2ball_reduction():
    """proj_ellipse_fb solves min (z-s)^H diag(1/pU) (z-s) s.t. ||z-y|| <= eps:
    on the sphere its KKT condition is (s - z)/pU = lam (z - y), lam >= 0; with
    pU = 1 one iteration is the l2-ball projection; inside the ball z = s."""
    rng = np.random.default_rng(4)
    n = 300
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    s = y + 3.0 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    pU = rng.uniform(0.2, 1.0, n)
    z, k = so.proj_ellipse_fb(s, y, pU, 10.0, np.zeros(n), max_itr=500, min_itr=1, stop=1e-12)
    assert abs(np.linalg.norm(z - y) - 10.0) < 1e-9
    lam = ((s - z) / pU) / (z - y)
    assert np.std(lam.real) < 1e-6 * abs(np.mean(lam.real)) and np.mean(lam.real) > 0
    assert np.max(np.abs(lam.imag)) < 1e-6
    z1, k1 = so.proj_ellipse_fb(s, y, np.ones(n), 10.0, np.zeros(n), 20, 1, 1e-10)
    assert np.allclose(z1, so.proj_l2ball(s, 10.0, y), atol=1e-12)
    zin, _ = so.proj_ellipse_fb(y + 0.01 * (s - y), y, pU, 10.0, np.zeros(n), 2000, 1, 1e-13)
    assert np.allclose(zin, y + 0.01 * (s - y), atol=1e-9)


def test_uniform_weight_preconditioner_counts():
    Ky = Kx = 16
    # three points in cell (1, 2), one in (0, 0), one on the wrapped edge (15 -> cell 15)
    g = 2 * np.pi / 16
    om_y = np.array([1 * g, 1.2 * g, 0.8 * g, 0.0, -1 * g])
    om_x = np.array([2 * g, 2.3 * g, 1.9 * g, 0.1 * g, 0.0])
    pU = so.uniform_weight_preconditioner(om_y, om_x, Ky, Kx)
    assert np.allclose(pU, [1 / 3, 1 / 3, 1 / 3, 1.0, 1.0])


def test_dr_operator_equals_gram_on_active_cells():
    """util_load_data_gen_dr_measurement_operator.m: the tril / half-diagonal
    H applied as H u + (u'H)' is G'G on the active cells; Lambda normalises
    diag(G'G) to 1; the DR matrix form equals the istril formulas."""
    from oracle import dr
    data, x, meta = problem.make_problem(16, 24, 1, 700, 3, seed=5, synth=synth)
    G = data.G[0]
    H, W, lam = dr.dr_operator(G, data.op.No)
    Gfull = sum((Gb.conj().T @ Gb) for Gb in G).toarray()
    assert np.array_equal(W, np.diag(Gfull).real > 0)
    assert 0 < W.sum() < W.size
    Hf = (H + H.conj().T).toarray()
    assert np.allclose(Hf, Gfull[np.ix_(W, W)], rtol=0, atol=1e-12 * np.abs(Gfull).max())
    assert np.allclose(lam ** 2 * np.diag(Hf).real, 1.0)
    rng = np.random.default_rng(0)
    Fx = rng.standard_normal(data.op.No) + 1j * rng.standard_normal(data.op.No)
    y = dr.dr_forward(H, lam, Fx[W])
    Gdr = dr.dr_matrix(H, W, lam)
    assert np.allclose(Gdr @ Fx, y)
    assert np.allclose(y, lam * (Gfull @ Fx)[W])
    v = rng.standard_normal(W.sum()) + 1j * rng.standard_normal(W.sum())
    g = np.zeros(data.op.No, dtype=complex)
    g[W] = dr.dr_adjoint(H, lam, v)
    assert np.allclose(Gdr.conj().T @ v, g)
    # coupling stays within the 13 x 13 stencil of two 7 x 7 supports
    Ky = data.op.Ky
    idx = np.flatnonzero(W)
    r, c = np.nonzero(np.abs(Hf) > 0)
    d0 = (idx[c] % Ky - idx[r] % Ky + Ky // 2) % Ky - Ky // 2
    d1 = (idx[c] // Ky - idx[r] // Ky + data.op.Kx // 2) % data.op.Kx - data.op.Kx // 2
    assert np.abs(d0).max() <= 6 and np.abs(d1).max() <= 6


def test_dr_reduced_data_and_dual_step():
    """The DR dual step of update_dual_data_fidelity.m:85-125 (istril branch,
    literal formulas) equals the oracle's l2-ball step on the DR data term."""
    from oracle import dr
    data, x, meta = problem.make_problem(16, 16, 2, 500, 2, seed=8, synth=synth)
    ddr, ops = dr.dr_data_term(data)
    rng = np.random.default_rng(3)
    v2 = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in ddr.y]
    Fx_old = np.stack([data.op.A(0.7 * x[l]) for l in range(2)])
    s22 = np.array([0.4, 0.3])
    out = so.update_dual_data_fidelity(v2, 0.9 * x, Fx_old, ddr, s22)
    for l, (H, W, lam) in enumerate(ops):
        Fx = data.op.A(0.9 * x[l])
        fp = 2 * Fx[W] - Fx_old[l][W]
        z = v2[l][0] + dr.dr_forward(H, lam, fp) - ddr.y[l][0]
        v2l = z * (1 - min(ddr.eps[l][0] / np.linalg.norm(z), 1))
        assert np.allclose(out[0][l][0], v2l)
        g2 = np.zeros(data.op.No, dtype=complex)
        g2[W] = dr.dr_adjoint(H, lam, v2l)
        assert np.allclose(out[1][l], s22[l] * np.real(data.op.At(g2)))
        assert np.isclose(out[3][l][0], np.linalg.norm(dr.dr_forward(H, lam, Fx[W]) - ddr.y[l][0]))


def test_noise_adjustment_rule_and_trigger():
    """facetHyperSARA.m:883-944: eps_b grows to (eps_b + ||res_b||) c where
    eps_b < (2 - tol) ||res_b||; FHS adjusts at the run's first iteration,
    HS at adjust_noise_start_iter; priors stay off until then."""
    p = so.SolverParams(pdfb_fidelity_tolerance=1.01, adjust_noise_change_percentage=0.5)
    eps, sig = so.adjust_noise([[1.0, 5.0], [2.0]], [[3.0, 4.0], [1.0]], [[10, 30], [5]], p)
    assert eps == [[2.0, 5.0], [2.0]]                  # 1 < 0.99*3: raised; 5 >= 0.99*4 and 2 >= 0.99: kept
    assert np.allclose(sig, [np.sqrt((4 + 25) / 40), np.sqrt(4 / 5)])
    assert so.adjust_noise_trigger("fhs", 1, 0, 0.0, 10.0, 1.0, p)
    assert not so.adjust_noise_trigger("hs", 1, 0, 0.0, 10.0, 1.0, p)
    assert not so.adjust_noise_trigger("fhs", 1, 0, 0.0, 1.0, 1.0, p)   # residual within the bound
    Ny = Nx = 32
    data, x, meta = problem.make_problem(Ny, Nx, 2, 800, 2, seed=5, synth=synth)
    nu2 = so.operator_norm(data, 100, 1e-10)
    geom = FacetGeometry(Ny, Nx, 2, 2, (4, 4))
    sig, sig_bar, *_ = so.compute_noise_level(Ny, Nx, 2, np.ones(2), "fhs", geom, nu2)
    data.eps = [[0.3 * e for e in el] for el in data.eps]
    kw = dict(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
              pdfb_min_iter=10 ** 6, pdfb_max_iter=8, reweighting_flag=False)
    xa, loga = so.facet_hypersara(data, so.SolverParams(**kw, adjust_flag_noise=True), geom, max_iter=12)
    xb, logb = so.facet_hypersara(data, so.SolverParams(**kw), geom, max_iter=12)
    assert loga.n_adjust >= 1 and loga.epsilon[1] > 10 * loga.epsilon[0]
    assert all(e1 >= e0 for el0, el1 in zip(data.eps, loga.epsilon_final) for e0, e1 in zip(el0, el1))
    assert logb.epsilon[-1] == logb.epsilon[0] and not np.allclose(xa, xb)


def test_warm_start_network_layout_matches_the_oracle():
    """The product's U-Net layer list and parameter count equal the oracle's
    (the gradient check relies on one flat parameter layout)."""
    from fhs_b200 import warmstart
    from oracle import unet
    assert warmstart.layer_specs() == unet.layer_specs()
    assert warmstart.init_params().size == unet.n_params() == 2140065
