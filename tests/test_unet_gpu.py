"""The warm-start U-Net's hand-written kernels against the CPU oracle
(oracle/unet.py, PyTorch FP32 with the GPU's BF16 storage emulated).

Tolerances (BF16 activations and activation gradients, FP32 accumulation):
forward outputs 2e-2 relative; gradients 6e-2 relative per parameter tensor
(tensors holding at least 1e-3 of the gradient's norm) and a cosine of at
least 0.998 for the whole gradient.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FWD_TOL = 2e-2
GRAD_TOL = 6e-2
COS_MIN = 0.998


def _images(n, H, W, seed):
    """Smooth blobs and point sources, like the normalised dirty images."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W]
    out = np.zeros((n, H, W))
    for k in range(n):
        for _ in range(6):
            cy, cx, s = rng.uniform(0, H), rng.uniform(0, W), rng.uniform(1.5, 5)
            out[k] += rng.exponential(1.0) * np.exp(-0.5 * (((yy - cy) / s) ** 2 + ((xx - cx) / s) ** 2))
        out[k, rng.integers(0, H, 8), rng.integers(0, W, 8)] += rng.uniform(0.2, 1.0, 8)
        out[k] += 0.05 * rng.standard_normal((H, W))
    return out.astype(np.float32)


def _params(seed):
    from fhs_b200.warmstart import init_params
    p = init_params(seed)
    rng = np.random.default_rng(seed + 1)
    p += (0.01 * rng.standard_normal(p.size)).astype(np.float32)   # non-zero biases
    return p


def test_forward_matches_oracle():
    from fhs_b200.warmstart import UNet
    from helpers import rel
    from oracle import unet as ou
    import torch
    p = _params(3)
    im = _images(2, 32, 48, 5)
    net = UNet(params=p)
    out = net.forward(im)
    net.close()
    ref, _ = ou.forward(torch.tensor(p), im, bf16=True, dtype=torch.float32)
    assert rel(out, ref.detach().numpy()) < FWD_TOL


def test_gradient_matches_autograd():
    from fhs_b200.warmstart import UNet, layer_specs
    from oracle import unet as ou
    p = _params(4)
    im = _images(2, 32, 32, 6)
    tg = (0.7 * im + 0.1 * np.roll(im, 2, axis=2)).astype(np.float32)
    net = UNet(params=p)
    loss, g = net.gradient(im, tg)
    net.close()
    loss_o, g_o = ou.loss_and_grad(p, im, tg, bf16=True)
    assert abs(loss - loss_o) <= 2e-2 * abs(loss_o)
    cos = float(np.dot(g, g_o) / (np.linalg.norm(g) * np.linalg.norm(g_o)))
    assert cos >= COS_MIN, cos
    pos, gn = 0, np.linalg.norm(g_o)
    tensors = []
    for ci, co in layer_specs():
        tensors += [co * ci * 9, co]
    tensors += [32, 1]
    for k, n in enumerate(tensors):
        a, b = g[pos:pos + n], g_o[pos:pos + n]
        pos += n
        if np.linalg.norm(b) < 1e-3 * gn:
            continue
        assert np.linalg.norm(a - b) <= GRAD_TOL * np.linalg.norm(b), (k, np.linalg.norm(a - b) / np.linalg.norm(b))


def test_training_reduces_the_loss():
    """Adam steps of the library's kernels fit a fixed blur-and-shrink map."""
    from fhs_b200.warmstart import UNet, train
    im = _images(16, 32, 32, 7)
    tg = np.maximum(im - 0.1, 0.0).astype(np.float32)
    net = UNet(seed=1)
    losses = train(net, im, tg, steps=150, batch=8, lr=1e-3)
    net.close()
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-10:]) < 0.2 * np.mean(losses[:5]), (losses[:5], losses[-10:])
