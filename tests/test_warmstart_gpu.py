"""What the trained warm-start network gains over the cold start (GPU).

The network is trained by the library's own kernels on (dirty image,
plain-solver solution) pairs of seeded 64 x 64 x 4 HyperSARA cubes, then a
held-out cube is solved from its warm start and from zero: the warm start
must be used by the fallback rule, and after the same number of primal-dual
iterations (5 and 20) the warm-started iterate must have a reconstruction
SNR higher by at least 1 dB.  A network whose output is worse than zero must be
rejected by the fallback rule.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(seed, Ny=64, Nx=64, L=4):
    from fhs_b200 import heuristics, synth
    from fhs_b200.api import HS_forward_operator_G, MeasurementOperator
    rng = np.random.default_rng(seed)
    x = synth.sky_cube(Ny, Nx, L, seed)
    M = Ny * Nx // 2
    oy0, ox0 = synth.base_coverage(M, seed)
    nu = synth.frequencies(L)
    om = [synth.channel_coverage(oy0, ox0, nu[l], nu[-1]) for l in range(L)]
    bsz = [[M] for _ in range(L)]
    op0 = MeasurementOperator(Ny, Nx, om, bsz)
    y0 = HS_forward_operator_G(np.moveaxis(x, 0, 2), op0)
    op0.close()
    sig = [synth.noise_sigma(y0[l][0], 40.0) for l in range(L)]
    y = [[(y0[l][0] + sig[l] * synth.noise(M, rng)) / sig[l]] for l in range(L)]
    op = MeasurementOperator(Ny, Nx, om, bsz, [np.full(M, 1.0 / s) for s in sig])
    eps = [synth.l2_bounds(b) for b in bsz]
    nu2 = op.operator_norm(50, 1e-6)
    gam, gam0, *_ = heuristics.compute_noise_level(Ny, Nx, L, np.ones(L), "hs", nu2)
    param = dict(nu2=nu2, gamma=gam, gamma0=gam0, reweighting_sig=gam, reweighting_sig_bar=gam0,
                 pdfb_min_iter=10 ** 6, reweighting_flag=False)
    return x, op, y, eps, param


def _snr(x, xe):
    return 20 * np.log10(np.linalg.norm(x) / np.linalg.norm(x - xe))


@pytest.fixture(scope="module")
def trained():
    from fhs_b200 import warmstart as ws
    xin, xout = ws.training_pairs(16, 64, 64, 4, seed=100, pdfb_max_iter=200, reweighting_max_iter=1)
    net = ws.UNet(seed=2)
    losses = ws.train(net, xin, xout, steps=3000, batch=8, lr=1e-3)
    yield net, losses
    net.close()


def test_warm_start_beats_cold_start(trained):
    from fhs_b200 import warmstart as ws
    from fhs_b200._lib import ALGO_HS
    from fhs_b200.api import Solver
    net, losses = trained
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5])
    x, op, y, eps, param = _problem(555)
    x0, info = ws.warm_start(net, op, y, eps, param["gamma"], param["gamma0"])
    assert info["used"] and info["objective_warm"] < info["objective_cold"]
    out = {}
    for name, xinit in (("cold", None), ("warm", x0)):
        s = Solver(op, ALGO_HS, param)
        s.set_data(y, eps)
        s.init(xinit)
        done = 0
        for k in (1, 5, 20):
            s.iterate(k - done)
            done = k
            out[(name, k)] = _snr(np.moveaxis(x, 0, 2), s.x())
        s.close()
    op.close()
    print({f"{a}@{k}": round(v, 2) for (a, k), v in out.items()}, "x0:", round(_snr(np.moveaxis(x, 0, 2), x0), 2))
    # after one iteration both iterates equal their starting point (g = 0)
    for k in (5, 20):
        assert out[("warm", k)] > out[("cold", k)] + 1.0, out


def test_fallback_rejects_a_worse_start(trained):
    """A network scaled to return far too much flux loses to x = 0 on the
    objective, and the solver starts cold."""
    from fhs_b200 import warmstart as ws
    net, _ = trained
    p = net.params()
    bad = ws.UNet(params=p)
    q = p.copy()
    q[-33:-1] *= 1e3   # the 1x1 head weights
    bad.set_params(q)
    x, op, y, eps, param = _problem(556)
    x0, info = ws.warm_start(bad, op, y, eps, param["gamma"], param["gamma0"])
    bad.close()
    op.close()
    assert not info["used"] and not np.any(x0)


def test_device_warm_start_matches_the_host_route(trained):
    """fhs_solver_init_warm (every cube on the GPU) takes the same decision
    as the host route and starts from the same estimate: the dirty cubes
    differ at FP32 rounding level (hand-written vs library FFT), which the
    BF16 network passes on at the 2e-2 level of the network tests."""
    from fhs_b200 import warmstart as ws
    from fhs_b200._lib import ALGO_HS
    from fhs_b200.api import Solver
    from helpers import rel
    net, _ = trained
    x, op, y, eps, param = _problem(557)
    x0_h, info_h = ws.warm_start(net, op, y, eps, param["gamma"], param["gamma0"])
    s = Solver(op, ALGO_HS, param)
    s.set_data(y, eps)
    dec = ws.warm_start_device(net, s)
    assert dec["used"] == info_h["used"] and dec["used"]
    assert rel(s.x(), x0_h) < 2e-2
    assert abs(dec["objective_cold"] - info_h["objective_cold"]) < 1e-4 * info_h["objective_cold"]
    assert abs(dec["objective_warm"] - info_h["objective_warm"]) < 1e-2 * info_h["objective_warm"]
    s.iterate(5)   # the solver runs from the warm start
    assert _snr(np.moveaxis(x, 0, 2), s.x()) > _snr(np.moveaxis(x, 0, 2), x0_h)
    s.close()
    op.close()


def test_device_fallback_starts_from_zero(trained):
    from fhs_b200 import warmstart as ws
    from fhs_b200._lib import ALGO_HS
    from fhs_b200.api import Solver
    net, _ = trained
    q = net.params().copy()
    q[-33:-1] *= 1e3   # the 1x1 head weights
    bad = ws.UNet(params=q)
    x, op, y, eps, param = _problem(558)
    s = Solver(op, ALGO_HS, param)
    s.set_data(y, eps)
    dec = ws.warm_start_device(bad, s)
    bad.close()
    assert not dec["used"] and dec["objective_warm"] > dec["objective_cold"]
    assert not np.any(s.x())
    s.close()
    op.close()
