"""GPU update_dual_data_fidelity (pU = 1) vs the oracle, one step."""
import numpy as np
import pytest

from fhs_b200 import synth
from helpers import rel
from oracle import problem
from oracle import solvers as so

pytestmark = pytest.mark.gpu


def test_update_dual_data_fidelity_one_step():
    from fhs_b200 import MeasurementOperator, update_dual_data_fidelity
    data, x, meta = problem.make_problem(48, 48, 3, 2500, 3, seed=9, synth=synth)
    op = MeasurementOperator(48, 48, meta["om"], meta["blocks"],
                             [np.full(len(o[0]), 1.0 / s) for o, s in zip(meta["om"], meta["sigma"])])
    rng = np.random.default_rng(1)
    v2 = [[10.0 * (rng.standard_normal(len(b)) + 1j * rng.standard_normal(len(b))) for b in yl] for yl in data.y]
    xk = x * 0.9  # v2 large enough that z leaves the l2 ball (non-trivial update)
    Fx_old = np.stack([data.op.A(x[l] * 0.8) for l in range(3)])
    sigma22 = np.array([0.3, 0.2, 0.1])
    ref = so.update_dual_data_fidelity(v2, xk, Fx_old, data, sigma22)
    out = update_dual_data_fidelity(v2, data.y, np.moveaxis(xk, 0, 2), Fx_old.T, op, data.eps, sigma22)
    v2g, Ftx, Fx_new, norm_res, gres, geps = out
    for l in range(3):
        assert rel(np.concatenate(v2g[l]), np.concatenate(ref[0][l])) < 1e-5
        assert rel(Fx_new[:, l], ref[2][l]) < 1e-5
        assert np.allclose(norm_res[l], ref[3][l], rtol=1e-5)
    assert rel(np.moveaxis(Ftx, 2, 0), ref[1]) < 1e-5
    assert abs(gres - ref[4]) / ref[4] < 1e-5 and abs(geps - ref[5]) / ref[5] < 1e-12
