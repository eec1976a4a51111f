"""CPU oracle of the preconditioner network (TEST INFRASTRUCTURE).

The network has no counterpart in the reference (whose tomography CG,
src/ptychotomo/solver.py:180-203, is unpreconditioned); this file restates,
in float64 NumPy, what the project's CUDA kernels compute, so that their
forward values and parameter gradients can be checked:

    h1 = silu(W1 x + b1)        x in R^3, W1 [64, 3]
    h2 = silu(W2 h1 + b2)       W2 [64, 64]
    z  = W3 h2 + b3             W3 [64], b3 scalar
    loss = sum_p w_p (z_p - y_p)^2 * inv_wsum

with silu(s) = s / (1 + exp(-s)).  Parameters are one flat float32 vector
in the order W1 (row-major), b1, W2 (row-major), b2, W3, b3 (4481 values).
With ``bf16=True`` the weights (not the biases) are first rounded to
bfloat16, round-to-nearest-even, as the kernels do before their FP32
arithmetic.
"""
from __future__ import annotations

import numpy as np

H, DIN = 64, 3
SHAPES = (("W1", (H, DIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H,)), ("b3", (1,)))
NPAR = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(params):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def bf16_round(a):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    b = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def effective(params, bf16=True):
    """The parameter values the arithmetic uses (float64; the weights rounded
    to bfloat16 from their float32 values when bf16)."""
    p = np.asarray(params, np.float64).copy()
    if bf16:
        d = unpack(p)
        for k in ("W1", "W2", "W3"):
            d[k] = bf16_round(d[k].astype(np.float32)).astype(np.float64)
        p = pack(d)
    return p


def _silu(s):
    return s / (1.0 + np.exp(-s))


def _dsilu(s):
    sg = 1.0 / (1.0 + np.exp(-s))
    return sg * (1.0 + s * (1.0 - sg))


def forward(params, x, bf16=True, act_bf16=False):
    """act_bf16: the hidden layer h1 enters the 64 x 64 layer rounded to
    bfloat16 (from its float32 value), as in the tensor-core forward."""
    d = unpack(effective(params, bf16))
    x = np.asarray(x, np.float64).reshape(-1, DIN)
    s1 = x @ d["W1"].T + d["b1"]
    h1 = _silu(s1)
    if act_bf16:
        h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    s2 = h1 @ d["W2"].T + d["b2"]
    return _silu(s2) @ d["W3"] + d["b3"][0]


def loss_and_grad(params, x, y, w, inv_wsum, bf16=True):
    """Loss and its gradient with respect to the (effective) parameters."""
    d = unpack(effective(params, bf16))
    x = np.asarray(x, np.float64).reshape(-1, DIN)
    y = np.asarray(y, np.float64)
    w = np.asarray(w, np.float64)
    s1 = x @ d["W1"].T + d["b1"]
    h1 = _silu(s1)
    s2 = h1 @ d["W2"].T + d["b2"]
    h2 = _silu(s2)
    z = h2 @ d["W3"] + d["b3"][0]
    r = z - y
    loss = float(np.sum(w * r * r) * inv_wsum)
    dz = 2.0 * w * r * inv_wsum
    g = {"W3": h2.T @ dz, "b3": np.array([dz.sum()])}
    ds2 = np.outer(dz, d["W3"]) * _dsilu(s2)
    g["W2"] = ds2.T @ h1
    g["b2"] = ds2.sum(0)
    ds1 = (ds2 @ d["W2"]) * _dsilu(s1)
    g["W1"] = ds1.T @ x
    g["b1"] = ds1.sum(0)
    return loss, pack(g)


def adam(params, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba, 2015) with bias correction, in float64."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
