"""GPU nuclear norm and l2-ball projection vs the oracle (FP64 reference)."""
import numpy as np
import pytest

from oracle import solvers as so

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [1, 3, 16, 20, 33, 64])
def test_nuclear_norm(L):
    from fhs_b200 import nuclear_norm
    rng = np.random.default_rng(L)
    x = rng.standard_normal((40, 24, L)) + np.outer(rng.random(40 * 24), rng.random(L)).reshape(40, 24, L) * 5
    ref = so.nuclear_norm(np.moveaxis(x, 2, 0))
    assert abs(nuclear_norm(x) - ref) / ref < 1e-5


@pytest.mark.parametrize("scale", [0.1, 10.0])
def test_proj_l2ball(scale):
    from fhs_b200 import proj_l2ball
    rng = np.random.default_rng(3)
    y = rng.standard_normal(1000) + 1j * rng.standard_normal(1000)
    x = y + scale * (rng.standard_normal(1000) + 1j * rng.standard_normal(1000))
    eps = 30.0
    p = proj_l2ball(x, eps, y)
    assert np.allclose(p, so.proj_l2ball(x, eps, y), rtol=1e-12, atol=1e-12)
    assert np.linalg.norm(p - y) <= eps * (1 + 1e-12)


def test_nuclear_norm_nearly_low_rank_cube():
    """A power-law spectral cube is nearly low rank: its small singular values
    need the FP64 Gram (an FP32-accurate Gram misses them by ~sqrt(1e-7)
    sigma_max; measured 4.9e-4 relative on the nuclear norm at 2048^2 x 32)."""
    from fhs_b200 import nuclear_norm, synth
    x = synth.sky_cube(256, 256, 32, 9)
    ref = so.nuclear_norm(x)
    assert abs(nuclear_norm(np.moveaxis(x, 0, 2)) - ref) / ref < 1e-6, (nuclear_norm(np.moveaxis(x, 0, 2)), ref)
