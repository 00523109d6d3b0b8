"""CPU restatement of the GPU MLP (lbib_mlp_*), the checker of its
forward pass and gradients.  Test infrastructure only.

Same model as the kernels: per layer Z = A W^T + b with A and W rounded to
bfloat16 (round to nearest even), GELU (erf form) after every layer but
the last, whose activations are rounded to bfloat16 again; loss = mean of
(Y - T)^2 over batch and outputs; the backward pass rounds dY and every dZ
to bfloat16 as the kernels store them.  Accumulation here is FP64 (the GPU
accumulates in FP32).  With round=False everything stays FP64 -- the form
the finite-difference check uses.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params, widths):
    out, i = [], 0
    for l in range(len(widths) - 1):
        n_in, n_out = widths[l], widths[l + 1]
        W = np.asarray(params[i:i + n_in * n_out], dtype=np.float64).reshape(n_out, n_in)
        i += n_in * n_out
        b = np.asarray(params[i:i + n_out], dtype=np.float64)
        i += n_out
        out.append((W, b))
    return out


def forward(params, widths, X, round=True):
    r = bf16 if round else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params, widths)
    A = [r(X)]
    Z = []
    for l, (W, b) in enumerate(layers):
        z = A[-1] @ r(W).T + b
        Z.append(z)
        if l + 1 < len(layers):
            A.append(r(gelu(z)))
    return Z[-1], A, Z


def loss_and_grad(params, widths, X, T, round=True):
    r = bf16 if round else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params, widths)
    Y, A, Z = forward(params, widths, X, round)
    B, w = T.shape
    loss = float(np.mean((Y - T) ** 2))
    dZ = r(2.0 * (Y - T) / (B * w))
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        grads[l] = (dZ.T @ A[l], dZ.sum(axis=0))
        if l == 0:
            break
        dA = dZ @ r(W)
        dZ = r(dA * gelu_grad(Z[l - 1]))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
