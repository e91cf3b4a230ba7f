"""CPU restatement of the learned surrogate (test infrastructure only: the tests use it as the checker
of the library's tensor-core forward and backward kernels; nothing in the library calls it).

The network has no counterpart in the reference. Layout of the parameter vector theta:
W[4][64][64] (out x in), b[4][64], w5[64], b5. The arithmetic follows the GPU kernels' roundings:
the features and every hidden activation enter a layer as BF16 (round to nearest even), the hidden
weights are BF16, products are accumulated in higher precision here (FP32 on the GPU), the biases,
activations and the output layer are FP32/FP64. Backward: dZ enters both the weight-gradient and the
input-gradient products as BF16; the bias gradients sum the unrounded dZ.
"""
from __future__ import annotations

import numpy as np

NF = 32
W = 64
NL = 4
NW = NL * W * W
NPARAM = NW + NL * W + W + 1


def bf16(x):
    """Rounds float32 values to bfloat16 (nearest even); returns float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(theta):
    theta = np.asarray(theta)
    Wl = theta[:NW].reshape(NL, W, W)
    b = theta[NW:NW + NL * W].reshape(NL, W)
    w5 = theta[NW + NL * W:NW + NL * W + W]
    b5 = theta[NW + NL * W + W]
    return Wl, b, w5, b5


def features(pts, freq, io):
    """[sin(2 pi B x_n), cos(2 pi B x_n)] with x_n = (p - centre) * scale."""
    io = np.asarray(io, np.float64)
    xn = (np.asarray(pts, np.float32).astype(np.float64) - io[:3]) * io[3:6]
    t = 2.0 * np.pi * (xn @ np.asarray(freq, np.float64).reshape(NF, 3).T)
    return np.concatenate([np.sin(t), np.cos(t)], axis=1)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def forward(pts, theta, freq, io, cache=False, rounding=True):
    """f_net at pts; rounding=False skips the BF16 roundings (the smooth function the kernels approximate)."""
    r = (lambda x: bf16(x).astype(np.float64)) if rounding else (lambda x: np.asarray(x, np.float64))
    Wl, b, w5, b5 = unpack(theta)
    Wb = r(Wl)
    h = r(features(pts, freq, io))
    ins, zs = [], []
    a = None
    for l in range(NL):
        ins.append(h)
        z = h @ Wb[l].T + b[l]
        zs.append(z)
        a = _silu(z)
        h = r(a)
    f = a @ w5.astype(np.float64) + float(b5)
    if cache:
        return f, (Wb, ins, zs, a)
    return f


def gradient(pts, targets, theta, freq, io, rounding=True):
    """Gradient of mean((f - clamp(target))^2) and the loss, in the parameter layout above."""
    r = (lambda x: bf16(x).astype(np.float64)) if rounding else (lambda x: np.asarray(x, np.float64))
    Wl, b, w5, b5 = unpack(theta)
    f, (Wb, ins, zs, a4) = forward(pts, theta, freq, io, cache=True, rounding=rounding)
    c = float(io[6])
    t = np.clip(np.asarray(targets, np.float64), -c, c)
    n = len(f)
    e = f - t
    loss = float(np.mean(e * e))
    g = 2.0 * e / n
    grad = np.zeros(NPARAM, np.float64)
    grad[NW + NL * W:NW + NL * W + W] = a4.T @ g
    grad[-1] = g.sum()
    dh = np.outer(g, w5.astype(np.float64))
    for l in range(NL - 1, -1, -1):
        z = zs[l]
        s = 1.0 / (1.0 + np.exp(-z))
        dz = dh * s * (1.0 + z * (1.0 - s))
        grad[NW + l * W:NW + (l + 1) * W] = dz.sum(0)
        dzb = r(dz)
        grad[l * W * W:(l + 1) * W * W] = (dzb.T @ ins[l]).reshape(-1)
        if l > 0:
            dh = dzb @ Wb[l]
    return grad, loss


def random_params(seed, freq_sigma=4.0):
    """Parameters drawn like the library's initialisation (uniform +-1/8, Gaussian frequencies)."""
    rng = np.random.default_rng(seed)
    theta = rng.uniform(-0.125, 0.125, NPARAM).astype(np.float32)
    freq = rng.normal(0.0, freq_sigma, (NF, 3)).astype(np.float32)
    return theta, freq
