"""GPU SARA dictionary (db1..db8 + Dirac, 4 levels, zero padding) vs the oracle.

Tolerances: coefficients and syntheses within 1e-5 relative of the FP64
oracle; the GPU transform pair is adjoint and perfectly reconstructing to 1e-6.
"""
import numpy as np
import pytest

from helpers import rel
from oracle import wavelets as wv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Ny,Nx,L", [(64, 64, 2), (37, 29, 3), (128, 96, 1), (16, 20, 2)])
def test_analysis_synthesis_match_oracle(Ny, Nx, L):
    from fhs_b200 import sara_analysis, sara_n_coefs, sara_synthesis
    rng = np.random.default_rng(Ny + Nx)
    x = rng.standard_normal((Ny, Nx, L))
    c = sara_analysis(x)
    assert c.shape == (wv.n_coefs_sara(Ny, Nx), L) and sara_n_coefs(Ny, Nx) == c.shape[0]
    co = wv.sara_analysis(np.moveaxis(x, 2, 0))
    assert rel(c.T, co) < 1e-5
    cc = rng.standard_normal(c.shape)
    xs = sara_synthesis(cc, Ny, Nx)
    xo = wv.sara_synthesis(cc.T, Ny, Nx)
    assert rel(np.moveaxis(xs, 2, 0), xo) < 1e-5
    # adjoint pair and perfect reconstruction of the GPU transforms
    assert abs(np.sum(c * cc) - np.sum(x * xs)) / abs(np.sum(c * cc)) < 1e-5
    assert rel(sara_synthesis(c, Ny, Nx), x) < 1e-6


def test_sara_prior_matches_oracle():
    from fhs_b200 import compute_sara_prior
    from oracle.solvers import compute_sara_prior as ref
    x = np.abs(np.random.default_rng(5).standard_normal((48, 40, 4)))
    assert abs(compute_sara_prior(x) - ref(np.moveaxis(x, 2, 0))) / ref(np.moveaxis(x, 2, 0)) < 1e-5
