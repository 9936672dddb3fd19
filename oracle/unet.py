"""CPU reference of the warm-start U-Net (test infrastructure only).

The checker for the library's BF16 U-Net kernels (``fhs_unet_*``): the same
architecture and parameter layout in PyTorch on the CPU (FP32 or FP64), whose
autograd gradients check the library's hand-written backward kernels.  With
``bf16=True`` the weights and every activation map are rounded to bfloat16 as
the GPU stores them (the arithmetic stays FP32), which isolates the kernels'
own error from the storage format's.

Architecture (4 levels, 32 base channels): encoder levels of two 3x3
convolutions + ReLU (32, 64, 128, 256 channels) with 2x2 average pooling in
between; decoder levels of a nearest 2x upsample, a 3x3 convolution + ReLU,
concatenation with the encoder map of the level, and two 3x3 convolutions +
ReLU; a 1x1 convolution to one channel.  Inputs are scaled by
s = 1 / max|image| per image; the output is divided by s again.
The loss is mean((s (out - target))^2) over all pixels.
"""
from __future__ import annotations

import numpy as np


def layer_specs(b=32):
    return [(1, b), (b, b), (b, 2 * b), (2 * b, 2 * b), (2 * b, 4 * b), (4 * b, 4 * b), (4 * b, 8 * b),
            (8 * b, 8 * b), (8 * b, 4 * b), (8 * b, 4 * b), (4 * b, 4 * b), (4 * b, 2 * b), (4 * b, 2 * b),
            (2 * b, 2 * b), (2 * b, b), (2 * b, b), (b, b)]


def n_params(b=32):
    return sum(co * ci * 9 + co for ci, co in layer_specs(b)) + b + 1


def init_params(seed=0, b=32):
    """He-normal weights, zero biases, head weight small (outputs start near 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in layer_specs(b):
        out.append(rng.standard_normal(co * ci * 9) * np.sqrt(2.0 / (ci * 9)))
        out.append(np.zeros(co))
    out.append(rng.standard_normal(b) * 1e-2)
    out.append(np.zeros(1))
    return np.concatenate(out).astype(np.float32)


def split_params(flat, b=32):
    import torch
    t = torch.as_tensor(flat)
    pos, layers = 0, []
    for ci, co in layer_specs(b):
        w = t[pos:pos + co * ci * 9].reshape(co, ci, 3, 3)
        pos += co * ci * 9
        bias = t[pos:pos + co]
        pos += co
        layers.append((w, bias))
    hw = t[pos:pos + b].reshape(1, b, 1, 1)
    pos += b
    hb = t[pos:pos + 1]
    return layers, hw, hb


def forward(params, images, b=32, bf16=False, dtype=None):
    """params: torch tensor (requires_grad allowed); images [n, H, W] numpy.
    Returns (out [n, H, W] tensor, scale [n])."""
    import torch
    import torch.nn.functional as F
    dtype = dtype or params.dtype
    img = torch.as_tensor(np.asarray(images), dtype=dtype)
    m = img.abs().amax(dim=(1, 2))
    s = torch.where(m > 0, 1.0 / m, torch.ones_like(m))
    x = (img * s[:, None, None])[:, None]

    def r(t):
        return t.to(torch.bfloat16).to(dtype) if bf16 else t

    layers, hw, hb = split_params(params, b)
    layers = [(r(w), bb) for w, bb in layers]

    def conv(t, k, relu=True):
        w, bb = layers[k]
        y = F.conv2d(t, w, bb, padding=1)
        return r(F.relu(y) if relu else y)

    def pool(t):
        return r(F.avg_pool2d(t, 2))

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    x = r(x)
    e1 = conv(conv(x, 0), 1)
    e2 = conv(conv(pool(e1), 2), 3)
    e3 = conv(conv(pool(e2), 4), 5)
    bb_ = conv(conv(pool(e3), 6), 7)
    u3 = conv(up(bb_), 8)
    d3 = conv(conv(torch.cat([u3, e3], 1), 9), 10)
    u2 = conv(up(d3), 11)
    d2 = conv(conv(torch.cat([u2, e2], 1), 12), 13)
    u1 = conv(up(d2), 14)
    d1 = conv(conv(torch.cat([u1, e1], 1), 15), 16)
    head = F.conv2d(d1, hw, hb)[:, 0]
    out = head / s[:, None, None]
    return out, s


def loss_and_grad(flat, images, targets, b=32, bf16=False, dtype=None):
    """(loss, gradient) by autograd."""
    import torch
    dtype = dtype or torch.float32
    p = torch.tensor(np.asarray(flat, dtype=np.float64), dtype=dtype, requires_grad=True)
    out, s = forward(p, images, b, bf16, dtype)
    tgt = torch.as_tensor(np.asarray(targets), dtype=dtype)
    e = (out - tgt) * s[:, None, None]
    loss = (e * e).mean()
    loss.backward()
    return float(loss.detach()), p.grad.detach().numpy().astype(np.float64)
