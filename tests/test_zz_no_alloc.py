"""The allocation-free l2-ball projection (fhs_proj_l2ball_noalloc).

Some callers cannot allocate device memory (hosts whose own pool owns the
device heap, real-time pipelines that forbid allocation after start-up); this
entry point takes device buffers and
keeps its partial sums in a static device array.  The test calls it through
the C ABI twice in a row, with different sizes and inputs, and checks each
result against fhs_proj_l2ball (the allocating entry point) to the 1e-12
tolerance of the projection tests.  It lives in its own file so that pytest
collects it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _device_array(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a.view(np.float64))).to("cuda:0")


@pytest.mark.parametrize("n1,n2", [(1000, 300001), (70000, 5)])
def test_noalloc_matches_allocating_entry_point(n1, n2):
    torch = pytest.importorskip("torch")
    from fhs_b200._lib import check, lib
    from fhs_b200 import proj_l2ball
    rng = np.random.default_rng(n1 + n2)
    for n, scale, eps in ((n1, 10.0, 3.0), (n2, 0.01, 50.0)):
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        x = y + scale * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
        xd, yd = _device_array(torch, x), _device_array(torch, y)
        pd = torch.empty_like(xd)
        stream = torch.cuda.current_stream(0).cuda_stream
        check(lib().fhs_proj_l2ball_noalloc(0, n, xd.data_ptr(), eps, yd.data_ptr(), pd.data_ptr(), stream))
        torch.cuda.synchronize(0)
        p = pd.cpu().numpy().view(np.complex128)
        ref = proj_l2ball(x, eps, y)
        assert np.allclose(p, ref, rtol=TOL, atol=TOL)


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    from fhs_b200._lib import FhsError, check, lib
    buf = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    with pytest.raises(FhsError, match="static scratch limit"):
        check(lib().fhs_proj_l2ball_noalloc(0, 1 << 40, buf.data_ptr(), 1.0, buf.data_ptr(), buf.data_ptr(), None))

