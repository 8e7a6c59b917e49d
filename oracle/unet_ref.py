"""PyTorch-CPU FP64 restatement of the warm-start U-Net (test infrastructure).

It mirrors musoc_solver_b200/unet.py layer for layer and rounds every stored
activation to BF16 as the GPU kernels do (weights are the GPU's BF16 working
copies), so that the GPU forward output and the autograd gradients can be
compared with tolerances set by BF16 rounding only.  Used by tests only.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

CONVS = [("enc0a", 16, 32), ("enc0b", 32, 32), ("enc1a", 32, 64), ("enc1b", 64, 64),
         ("enc2a", 64, 128), ("enc2b", 128, 128), ("bota", 128, 256), ("botb", 256, 256),
         ("up2", 256, 128), ("dec2a", 256, 128), ("dec2b", 128, 128), ("up1", 128, 64),
         ("dec1a", 128, 64), ("dec1b", 64, 64), ("up0", 64, 32), ("dec0a", 64, 32),
         ("dec0b", 32, 32)]


class _RoundBF16(torch.autograd.Function):
    """Rounds a stored tensor to BF16 in the forward pass and the gradient
    that arrives at it in the backward pass (the GPU stores both in BF16)."""

    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).to(torch.float64)

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).to(torch.float64)


def rb(x):
    return _RoundBF16.apply(x)


def bf16_round(a: np.ndarray) -> np.ndarray:
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


def forward_backward(state: dict, x_nhwc: np.ndarray, target: np.ndarray):
    """state: {name.0: w[9][ci][co] FP32, name.1: bias, head.0: w[32], head.1: b[1]}.
    x_nhwc: (B, H, W, 16); target: (B*H*W,).  Returns y (flat), loss,
    and gradients {name.0, name.1} (FP64)."""
    P = {}
    for name, ci, co in CONVS:
        w = torch.tensor(bf16_round(state[f"{name}.0"]), requires_grad=True)
        b = torch.tensor(np.asarray(state[f"{name}.1"], np.float64), requires_grad=True)
        P[name] = (w, b)
    hw = torch.tensor(np.asarray(state["head.0"], np.float64), requires_grad=True)
    hb = torch.tensor(np.asarray(state["head.1"], np.float64), requires_grad=True)

    def conv(name, x):
        w, b = P[name]
        wt = w.reshape(3, 3, w.shape[1], w.shape[2]).permute(3, 2, 0, 1)  # co, ci, ky, kx
        return rb(F.relu(F.conv2d(x, wt, bias=b, padding=1)))

    x = torch.tensor(np.asarray(x_nhwc, np.float64)).permute(0, 3, 1, 2)
    e0a = conv("enc0a", x)
    e0b = conv("enc0b", e0a)
    p0 = rb(F.avg_pool2d(e0b, 2))
    e1a = conv("enc1a", p0)
    e1b = conv("enc1b", e1a)
    p1 = rb(F.avg_pool2d(e1b, 2))
    e2a = conv("enc2a", p1)
    e2b = conv("enc2b", e2a)
    p2 = rb(F.avg_pool2d(e2b, 2))
    b0 = conv("bota", p2)
    b1 = conv("botb", b0)
    u2 = rb(F.interpolate(b1, scale_factor=2, mode="nearest"))
    c2 = rb(torch.cat([conv("up2", u2), e2b], dim=1))
    d2 = conv("dec2b", conv("dec2a", c2))
    u1 = rb(F.interpolate(d2, scale_factor=2, mode="nearest"))
    c1 = rb(torch.cat([conv("up1", u1), e1b], dim=1))
    d1 = conv("dec1b", conv("dec1a", c1))
    u0 = rb(F.interpolate(d1, scale_factor=2, mode="nearest"))
    c0 = rb(torch.cat([conv("up0", u0), e0b], dim=1))
    d0 = conv("dec0b", conv("dec0a", c0))
    y = (d0 * hw.reshape(1, -1, 1, 1)).sum(dim=1) + hb
    y = y.reshape(-1)
    t = torch.tensor(np.asarray(target, np.float64))
    loss = ((y - t) ** 2).mean()
    loss.backward()
    grads = {}
    for name, _, _ in CONVS:
        grads[f"{name}.0"] = P[name][0].grad.numpy()
        grads[f"{name}.1"] = P[name][1].grad.numpy()
    grads["head.0"] = hw.grad.numpy()
    grads["head.1"] = hb.grad.numpy()
    return y.detach().numpy(), float(loss.item()), grads
