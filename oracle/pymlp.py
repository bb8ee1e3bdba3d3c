"""CPU reference of the chemistry surrogate's network: test infrastructure only (the GPU path never
imports it). It repeats the GPU's forward and backward pass in float64 with BF16 rounding at the
same places (inputs, weights, hidden activations, back-propagated errors), so that the library's
tensor-core gradients can be checked against it to FP32-accumulation accuracy.

Layer l has weights W_l (rows_l x cols_l) and biases b_l; rows = (256, 256, 256, 16), cols =
(16, 256, 256, 256); the parameter blob stores W_0, b_0, W_1, b_1, ... row-major.
"""
import math

import numpy as np

ROWS = (256, 256, 256, 16)
COLS = (16, 256, 256, 256)


def bf16(a):
    """Round float32 values to BF16 (round to nearest even), returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


K2 = 2.0 * math.sqrt(2.0 / math.pi)  # 2 sqrt(2 / pi)


def _tanh_u(x):
    """tanh(u), u = sqrt(2 / pi) (x + 0.044715 x^3)"""
    return np.tanh(0.5 * K2 * x * (1.0 + 0.044715 * x * x))


def gelu(x):
    """GELU in its tanh form, 0.5 x (1 + tanh(u)) (the GPU evaluates tanh in hardware)."""
    return 0.5 * x * (1.0 + _tanh_u(x))


def gelu_grad(x):
    t = _tanh_u(x)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * 0.5 * K2 * (1.0 + 3.0 * 0.044715 * x * x)


def unpack(blob):
    p, out = 0, []
    for r, c in zip(ROWS, COLS):
        W = np.asarray(blob[p:p + r * c], dtype=np.float32).reshape(r, c)
        p += r * c
        b = np.asarray(blob[p:p + r], dtype=np.float32)
        p += r
        out.append((W, b))
    return out


def loss_and_grads(params, x, t, nout):
    """Mean squared error over the first nout output columns and its gradients (list of (gW, gb))."""
    B = x.shape[0]
    Wb = [bf16(W) for W, _ in params]
    bs = [b.astype(np.float64) for _, b in params]
    a = bf16(x)
    pres, hs = [], []
    for l in range(3):
        pre = (a @ Wb[l].T + bs[l]).astype(np.float32).astype(np.float64)
        h = bf16(gelu(pre))
        pres.append(pre)
        hs.append(h)
        a = h
    out = a @ Wb[3].T + bs[3]
    d = out - t
    d[:, nout:] = 0.0
    loss = float((d[:, :nout] ** 2).sum() / (B * nout))
    g = 2.0 * d / (B * nout)
    gb_ = bf16(g)
    grads = [None] * 4
    grads[3] = (gb_.T @ hs[2], g.sum(axis=0))
    dz = (gb_ @ Wb[3]) * gelu_grad(pres[2])
    for l in (2, 1, 0):
        dzb = bf16(dz)
        inp = hs[l - 1] if l > 0 else bf16(x)
        grads[l] = (dzb.T @ inp, dz.sum(axis=0))
        if l > 0:
            dz = (dzb @ Wb[l]) * gelu_grad(pres[l - 1])
    return loss, grads
