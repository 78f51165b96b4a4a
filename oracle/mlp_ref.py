"""ORACLE -- TEST INFRASTRUCTURE ONLY.

CPU restatement (numpy, float64 sums) of the warm-start MLP's forward pass and of its
backward pass for the loss mean((y - t)^2) over the rows and the 6 outputs, with the
same BF16 roundings as the device: weights, inputs, hidden activations and the
backpropagated gradients are rounded to BF16 where the device stores them in BF16;
everything is summed in float64 (the device sums in FP32 on the tensor cores).
"""
import numpy as np

NOUT = 6


ROUND = True      # the tests of the restatement itself switch the BF16 roundings off


def bf16(a):
    """Round float32/float64 values to the nearest BF16 (ties to even), returned as float64."""
    if not ROUND:
        return np.asarray(a, np.float64)
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(ws, X):
    """ws: [(W[out][in], b[out]) x 4] fp32; X: features [rows][64] (already bf16 values).
    Returns (y [rows][16] float64, hidden activations [H0=X, H1, H2, H3] as bf16 float64)."""
    H = [bf16(X)]
    for l in range(3):
        W, b = ws[l]
        a = H[-1] @ bf16(W).T + b.astype(np.float64)
        H.append(bf16(np.maximum(a, 0.0)))
    W, b = ws[3]
    y = H[-1] @ bf16(W).T + b.astype(np.float64)
    return y, H


def backward(ws, X, T):
    """Loss before any update and the gradients [(gT[in][out], gb[out]) x 4]."""
    y, H = forward(ws, X)
    rows = X.shape[0]
    e = np.zeros_like(y)
    e[:, :NOUT] = y[:, :NOUT] - T
    loss = float(np.sum(e[:, :NOUT] ** 2) / (rows * NOUT))
    dY = (2.0 / (rows * NOUT)) * e
    if ROUND:
        dY = dY.astype(np.float32).astype(np.float64)    # the device keeps dY in fp32
    grads = [None] * 4
    dZ = bf16(dY)
    gb_src = dY
    for l in range(3, -1, -1):
        W, _ = ws[l]
        gT = H[l].T @ dZ
        gb = gb_src.sum(0)
        grads[l] = (gT, gb)
        if l > 0:
            dH = dZ @ bf16(W)
            dZ = bf16(dH * (H[l] > 0))
            gb_src = dZ
    return loss, grads
