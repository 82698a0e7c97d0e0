"""CPU restatement (numpy, FP64 arithmetic) of the closure MLP's training
math -- TEST INFRASTRUCTURE ONLY, what the training kernels are tested against
(combustioncodegpu_b200/csrc/closure_train.cu); the product never calls it.

Network: n_in -> H -> H -> H -> n_out, SiLU on the hidden layers.
Quantisation-aware forward: every weight is rounded to BF16 (round to
nearest even) and the network inputs are BF16 values; the hidden activations
are FP32 (the inference kernel carries them as BF16 hi/lo pairs); the
backward pass treats the rounding as the identity (straight-through
estimator).  Loss: mean over batch and
outputs of ((o - y) * scale)^2.  Adam: Kingma & Ba (2015), bias-corrected.
Parameters: one flat array W1 [H][n_in], b1, W2 [H][H], b2, W3, b3,
W4 [n_out][H], b4.
"""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def layout(n_in, H, n_out):
    """[(offset of W, shape of W, offset of b, length of b)] per layer."""
    dims = [(H, n_in), (H, H), (H, H), (n_out, H)]
    out, o = [], 0
    for wo, wi in dims:
        out.append((o, (wo, wi), o + wo * wi, wo))
        o += wo * wi + wo
    return out, o


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(params, x, y, scale, n_in, H, n_out, quantized=True):
    """(loss, grad) of the quantisation-aware network on a batch
    (quantized=False: the same network without the BF16 rounding, in FP64,
    whose gradient a finite difference can check)."""
    lay, n = layout(n_in, H, n_out)
    r = (lambda v: bf16(v).astype(np.float64)) if quantized else (lambda v: np.asarray(v, dtype=np.float64))
    p = np.asarray(params, dtype=np.float32 if quantized else np.float64)
    W = [r(p[ow:ow + s[0] * s[1]].reshape(s)) for ow, s, _, _ in lay]
    b = [p[ob:ob + nb].astype(np.float64) for _, _, ob, nb in lay]
    a = [r(x)]  # rounded layer inputs
    z = []
    for l in range(4):
        zl = a[l] @ W[l].T + b[l]
        z.append(zl)
        if l < 3:
            a.append(_silu(zl).astype(np.float32).astype(np.float64) if quantized else _silu(zl))
    sc = np.asarray(scale, dtype=np.float64)
    err = (z[3] - np.asarray(y, dtype=np.float64)) * sc
    B = x.shape[0]
    loss = float(np.mean(err * err))
    g = 2.0 * err * sc / (B * n_out)
    grad = np.zeros(n)
    for l in range(3, -1, -1):
        ow, s, ob, nb = lay[l]
        grad[ow:ow + s[0] * s[1]] = (g.T @ a[l]).ravel()
        grad[ob:ob + nb] = g.sum(axis=0)
        if l > 0:
            g = (g @ W[l]) * _dsilu(z[l - 1])
    return loss, grad


def adam(params, grad, m, v, lr, beta1, beta2, eps, step):
    """One Adam step; returns (params, m, v)."""
    m = beta1 * m + (1.0 - beta1) * grad
    v = beta2 * v + (1.0 - beta2) * grad * grad
    c1, c2 = 1.0 - beta1 ** step, 1.0 - beta2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
