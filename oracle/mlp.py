"""The learned preconditioner's network restated in numpy (test infrastructure only).

Same network and loss as csrc/mlp.cu -- A1 = relu(X W1 + b1), A2 = relu(A1 W2 + b2),
Y = A2 W3 + b3, mean squared error against T -- with every GEMM operand rounded to
BF16 (round to nearest even) exactly where the kernel rounds it while staging, and
the products accumulated in FP64.  No counterpart in the reference.
Parameter order: W1 [in x H], b1, W2 [H x H], b2, W3 [H x out], b3 (row-major).
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, n_in, hid, n_out):
    p = np.asarray(params, np.float64)
    sizes = [n_in * hid, hid, hid * hid, hid, hid * n_out, n_out]
    out, o = [], 0
    for s in sizes:
        out.append(p[o:o + s])
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(n_in, hid), b1, W2.reshape(hid, hid), b2, W3.reshape(hid, n_out), b3


def _mm(a, b, exact):
    if exact:
        return np.asarray(a, np.float64) @ np.asarray(b, np.float64)
    return bf16(a) @ bf16(b)


def forward(params, X, n_in, hid, n_out, exact=False):
    """Activations A1, A2 and output Y; exact=True drops the BF16 rounding and keeps FP64 throughout."""
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, hid, n_out)
    cast = (lambda v: v) if exact else (lambda v: v.astype(np.float32))
    A1 = cast(np.maximum(_mm(X, W1, exact) + b1, 0.0))
    A2 = cast(np.maximum(_mm(A1, W2, exact) + b2, 0.0))
    Y = cast(_mm(A2, W3, exact) + b3)
    return A1, A2, Y


def gradients(params, X, T, n_in, hid, n_out, exact=False):
    """(loss, flat gradient) of the mean squared error."""
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, hid, n_out)
    A1, A2, Y = forward(params, X, n_in, hid, n_out, exact)
    cast = (lambda v: v) if exact else (lambda v: v.astype(np.float32))
    cnt = Y.size
    d = np.asarray(Y, np.float64) - T
    loss = float(np.sum(d * d) / cnt)
    dY = cast(2.0 * d / cnt)
    gW3 = _mm(A2.T, dY, exact)
    gb3 = np.asarray(dY, np.float64).sum(0)
    dZ2 = cast(np.where(A2 > 0, _mm(dY, W3.T, exact), 0.0))
    gW2 = _mm(A1.T, dZ2, exact)
    gb2 = np.asarray(dZ2, np.float64).sum(0)
    dZ1 = cast(np.where(A1 > 0, _mm(dZ2, W2.T, exact), 0.0))
    gW1 = _mm(np.asarray(X, np.float64 if exact else np.float32).T, dZ1, exact)
    gb1 = np.asarray(dZ1, np.float64).sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
