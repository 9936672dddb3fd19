"""GPU parity of the measurement operator against the FP64 oracle.

Tolerances: operator outputs within 1e-5 relative of the oracle (FP32 grid,
FFT and interpolation); the adjoint identity <Phi x, y> = <x, Phi^H y> of the
GPU operator within 1e-6 relative.
"""
import numpy as np
import pytest

from helpers import coverage, rel
from oracle.nufft import NufftOperator

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
ADJ_TOL = 1e-6


def _make(Ny, Nx, L, M, nblk, seed, weights=False):
    from fhs_b200 import MeasurementOperator
    om, bs, ws = [], [], []
    rng = np.random.default_rng(seed)
    for l in range(L):
        oy, ox = coverage(M + 17 * l, seed + l)
        om.append((oy, ox))
        sizes = [len(oy) // nblk] * (nblk - 1)
        sizes.append(len(oy) - sum(sizes))
        bs.append(sizes)
        ws.append(rng.uniform(0.5, 2.0, len(oy)) if weights else None)
    gop = MeasurementOperator(Ny, Nx, om, bs, ws)
    ref = NufftOperator(Ny, Nx)
    Gs = [ref.G(oy, ox, w) for (oy, ox), w in zip(om, ws)]
    return gop, ref, Gs


@pytest.mark.parametrize("Ny,Nx", [(64, 64), (48, 80), (16, 24), (128, 96)])
def test_scaled_fft_matches_oracle(Ny, Nx):
    gop, ref, _ = _make(Ny, Nx, 1, 200, 1, 1)
    x = np.random.default_rng(2).standard_normal((Ny, Nx))
    assert rel(gop.A(x), ref.A(x)) < OP_TOL
    Fx = ref.A(x)
    assert rel(gop.At(Fx), ref.At(Fx)) < OP_TOL


@pytest.mark.parametrize("Ny,Nx,M,nblk", [(64, 64, 3000, 2), (48, 80, 2500, 3), (16, 24, 300, 1),
                                         (256, 256, 40000, 4)])
def test_direct_adjoint_G_match_oracle(Ny, Nx, M, nblk):
    from fhs_b200 import apply_adjoint_operator, apply_direct_operator
    gop, ref, Gs = _make(Ny, Nx, 2, M, nblk, 11, weights=True)
    rng = np.random.default_rng(3)
    for l in range(2):
        Fx = rng.standard_normal(ref.No) + 1j * rng.standard_normal(ref.No)
        assert rel(apply_direct_operator(Fx, gop, l), Gs[l] @ Fx) < OP_TOL
        y = rng.standard_normal(Gs[l].shape[0]) + 1j * rng.standard_normal(Gs[l].shape[0])
        assert rel(apply_adjoint_operator(y, gop, l), Gs[l].conj().T @ y) < OP_TOL


def test_forward_adjoint_cube_and_adjointness():
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G
    Ny, Nx, L = 64, 64, 3
    gop, ref, Gs = _make(Ny, Nx, L, 4000, 3, 21)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((Ny, Nx, L))
    y = HS_forward_operator_G(x, gop)
    for l in range(L):
        yo = Gs[l] @ ref.A(x[:, :, l])
        assert rel(np.concatenate(y[l]), yo) < OP_TOL
    yr = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in y]
    xa = HS_adjoint_operator_G(yr, gop)
    for l in range(L):
        xo = np.real(ref.At(Gs[l].conj().T @ np.concatenate(yr[l])))
        assert rel(xa[:, :, l], xo) < OP_TOL
    # x is real, so the identity holds for Re<y, Phi x> = <Re(Phi^H y), x>
    lhs = sum(np.vdot(np.concatenate(yr[l]), np.concatenate(y[l])) for l in range(L)).real
    rhs = float(np.sum(xa * x))
    assert abs(lhs - rhs) / abs(lhs) < ADJ_TOL


def test_operator_norm_matches_oracle():
    from oracle.solvers import DataTerm, operator_norm
    gop, ref, Gs = _make(32, 32, 2, 1500, 1, 31)
    nu_gpu = gop.operator_norm(200, 1e-8)
    nu_ref = operator_norm(DataTerm(ref, [[G] for G in Gs], [[None]] * 2, [[1.0]] * 2), 200, 1e-10)
    assert np.allclose(nu_gpu, nu_ref, rtol=1e-4)


def test_compute_residual_images_matches_oracle():
    from fhs_b200 import compute_residual_images, synth
    from oracle import problem
    from oracle import solvers as so
    data, x, meta = problem.make_problem(48, 40, 3, 2000, 2, seed=13, synth=synth)
    from fhs_b200 import MeasurementOperator
    op = MeasurementOperator(48, 40, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    xk = 0.8 * x
    res = compute_residual_images(np.moveaxis(xk, 0, 2), data.y, op)
    ref = so.compute_residual_images(xk, data)
    assert rel(np.moveaxis(res, 2, 0), ref) < OP_TOL * 10


@pytest.mark.parametrize("Ny,Nx,L,M", [(32, 32, 2, 600), (64, 128, 2, 3000), (256, 128, 3, 8000),
                                       (512, 512, 2, 20000), (1024, 1024, 1, 40000), (2048, 2048, 1, 40000),
                                       (32, 2048, 1, 4000), (2048, 32, 1, 4000)])
def test_real_image_transforms_on_power_of_two_grids(Ny, Nx, L, M):
    """Phi x and Re(Phi^H y) of real images through the hand-written FFTs
    (every power-of-two grid side 64..4096, both axes, square and not)."""
    from fhs_b200 import HS_adjoint_operator_G, HS_forward_operator_G
    gop, ref, Gs = _make(Ny, Nx, L, M, 2, 41)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((Ny, Nx, L))
    y = HS_forward_operator_G(x, gop)
    for l in range(L):
        assert rel(np.concatenate(y[l]), Gs[l] @ ref.A(x[:, :, l])) < OP_TOL
    yr = [[rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b)) for b in yl] for yl in y]
    xa = HS_adjoint_operator_G(yr, gop)
    for l in range(L):
        xo = np.real(ref.At(Gs[l].conj().T @ np.concatenate(yr[l])))
        assert rel(xa[:, :, l], xo) < OP_TOL
    # relative to ||x|| ||Phi^H y|| (the Cauchy-Schwarz bound of both sides):
    # the sums cancel heavily for random vectors
    lhs = sum(np.vdot(np.concatenate(yr[l]), np.concatenate(y[l])) for l in range(L)).real
    assert abs(lhs - float(np.sum(xa * x))) / (np.linalg.norm(x) * np.linalg.norm(xa)) < ADJ_TOL
