"""The launch-shape autotuner (fhs_measop_autotune / set_tuning / tuning).

* the record: every candidate measured, the kept shapes among them;
* results do not depend on the shapes: FHS iterates with all FFT planes per
  launch and unsplit gridding items, and with 4-plane FFT chunks and
  1024-visibility gridding items (dense tiles split into partial tiles that
  a combine kernel sums), both within the 2e-5 iterate tolerance of the FP64
  oracle;
* changing the shapes between iterations makes the solver capture its
  iteration graph again: 2 iterations, a re-tuning, 3 more iterations match
  the oracle's 5;
* invalid shapes are refused.
"""
import numpy as np
import pytest

from helpers import rel
from test_solver_gpu import ITER_TOL, _gpu_solver, _oracle_run, _params, _setup

pytestmark = pytest.mark.gpu

SPLITS = ((0, 60, 128), (0, 70, 128))


def _problem():
    data, x, op, geom, nu2, sig, sig_bar = _setup("fhs", Ny=128, Nx=128, L=8, seed=9, overlap=(10, 10),
                                                  splits=SPLITS)
    param = _params(nu2, sig, sig_bar, pdfb_min_iter=10 ** 6, reweighting_flag=False)
    return data, op, geom, param


def test_autotune_record():
    _, op, _, _ = _problem()
    t = op.autotune()
    assert t["tuned"]
    assert set(t["fft_ms"]) == {0, 4}          # all planes, and chunks of 4 (< 8 channels)
    assert set(t["grid_ms"]) == {8192, 16384, 32768, 65536}
    assert all(v > 0 for v in list(t["fft_ms"].values()) + list(t["grid_ms"].values()))
    assert t["fft_chunk"] == min(t["fft_ms"], key=t["fft_ms"].get)
    assert t["grid_slice"] == min(t["grid_ms"], key=t["grid_ms"].get)
    assert op.tuning() == t
    op.close()


@pytest.mark.parametrize("shapes", [(0, 65536), (4, 1024)])
def test_iterates_do_not_depend_on_the_shapes(shapes):
    data, op, geom, param = _problem()
    op.set_tuning(*shapes)
    t = op.tuning()
    assert (t["fft_chunk"], t["grid_slice"]) == shapes and t["tuned"]
    s = _gpu_solver("fhs", op, param, geom, data)
    s.iterate(5)
    xo, _ = _oracle_run("fhs", data, param, geom, max_iter=5)
    assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL
    s.close()
    op.close()


def test_retuning_between_iterations():
    data, op, geom, param = _problem()
    op.set_tuning(0, 65536)
    s = _gpu_solver("fhs", op, param, geom, data)
    s.iterate(2)
    op.set_tuning(4, 1024)
    s.iterate(3)
    xo, _ = _oracle_run("fhs", data, param, geom, max_iter=5)
    assert rel(np.moveaxis(s.x(), 2, 0), xo) < ITER_TOL
    s.close()
    op.close()


def test_invalid_shapes_are_refused():
    _, op, _, _ = _problem()
    with pytest.raises(Exception):
        op.set_tuning(-1, 65536)
    with pytest.raises(Exception):
        op.set_tuning(0, 100)
    op.close()
