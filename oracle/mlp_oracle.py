"""CPU oracle for the sizing MLP's forward and backward pass.

TEST INFRASTRUCTURE ONLY (imported by tests/).  A plain numpy restatement of
the network in kmertreecounter_b200/csrc/kc_mlp.cu: three dense layers
(ReLU, ReLU, linear), batch-mean squared error, optionally weighted by
`under` where the output is below its target.  `bf16=True` rounds every
matrix-product operand to bfloat16 (round to nearest even) the way the GPU
kernels feed their tensor cores, and accumulates in float64; `bf16=False` is
the exact FP32-parameter reference the BF16 network approximates.
"""
import numpy as np


def to_bf16(x):
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


def forward_backward(x, t, layers, bf16=True, under=1.0):
    """layers = [(W0, b0), (W1, b1), (W2, b2)], W row-major fan_in x fan_out.
    Returns (y, loss, [(gW, gb) per layer])."""
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    W = [r(w) for w, _ in layers]
    bias = [np.asarray(b, np.float64) for _, b in layers]
    xb = r(x)
    h1 = np.maximum(xb @ W[0] + bias[0], 0.0)
    h1b = r(h1)
    h2 = np.maximum(h1b @ W[1] + bias[1], 0.0)
    h2b = r(h2)
    y = h2b @ W[2] + bias[2]
    n = y.size
    e = y - np.asarray(t, np.float64)
    w = np.where(e < 0, under, 1.0)
    loss = float((w * e * e).sum() / n)
    dy = 2.0 * w * e / n
    dyb = r(dy)
    g2 = (h2b.T @ dyb, dy.sum(0))
    dh2 = (dyb @ W[2].T) * (h2 > 0)
    dh2b = r(dh2)
    g1 = (h1b.T @ dh2b, dh2.sum(0))
    dh1 = (dh2b @ W[1].T) * (h1 > 0)
    dh1b = r(dh1)
    g0 = (xb.T @ dh1b, dh1.sum(0))
    return y, loss, [g0, g1, g2]
