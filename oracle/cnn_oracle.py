"""CPU restatement of the proposal network (test infrastructure only; the product path is the
tensor-core network in 3d-stereo-aldic_b200/csrc/cnn.cu).

The network has no counterpart in the reference (its initial guess is the integer search,
func/funIntegerSearch.m:132-180).  This module restates the device network in numpy so the
device's forward pass, gradients and training step can be checked:

  * rounding="bf16": the device's arithmetic points -- BF16 inputs, BF16 weight copies, BF16
    activations after each ReLU, BF16 output gradient and BF16 ReLU-masked gradients, with the
    products accumulated exactly (float64) where the device accumulates in FP32;
  * rounding=None: exact float64 math, pinned against central finite differences of the loss
    (tests/test_cnn_oracle.py), which checks the backward formulas themselves.

Layouts follow aldic_net_param_count(): per layer W (rows x cols, row-major) then b; conv K
ordered (ky, kx, channel); activations NHWC.
"""
from __future__ import annotations

import numpy as np

CONV = [(64, 2, 32, 18, 24), (32, 32, 32, 288, 288), (16, 32, 64, 288, 288), (8, 64, 64, 576, 576)]  # Hin Cin Cout K Kp
ROWS = [32, 32, 64, 64, 128, 16]
COLS = [24, 288, 288, 576, 1024, 128]
N_OUT, N_OUTP = 6, 16


def layout():
    """Offsets (w, b) of each layer in the flat parameter vector, and its length."""
    off, o = [], 0
    for r, c in zip(ROWS, COLS):
        off.append((o, o + r * c))
        o += r * c + r
    return off, o


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def init_params(seed=0):
    """He-normal weights, zero biases, zero padding columns / rows (FP32)."""
    off, n = layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    fan = [18, 288, 288, 576, 1024, 128]
    for l, (ow, ob) in enumerate(off):
        W = rng.normal(0.0, np.sqrt(2.0 / fan[l]), (ROWS[l], COLS[l])).astype(np.float32)
        if l == 0:
            W[:, 18:] = 0.0
        if l == 5:
            W[N_OUT:, :] = 0.0
        p[ow:ob] = W.ravel()
    return p


def _unpack(p):
    """Weights as float32 values (the device's FP32 master copy) in float64 arrays, or exact
    float64 parameters as they are."""
    off, _ = layout()
    return [(p[ow:ob].reshape(ROWS[l], COLS[l]), p[ob:ob + ROWS[l]]) for l, (ow, ob) in enumerate(off)]


def _im2col(H, Hin, Cin, K, Kp):
    """NHWC (B, Hin, Hin, Cin) -> (B * Hout^2, Kp): stride 2, pad 1, 3 x 3, K = (ky, kx, c)."""
    B = H.shape[0]
    Ho = Hin // 2
    Hp = np.zeros((B, Hin + 2, Hin + 2, Cin), dtype=H.dtype)
    Hp[:, 1:-1, 1:-1, :] = H
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(Hp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Ho:2, :])
    A = np.concatenate(cols, axis=3).reshape(B * Ho * Ho, K)
    if Kp > K:
        A = np.concatenate([A, np.zeros((A.shape[0], Kp - K), dtype=A.dtype)], axis=1)
    return A


def _col2im(dA, B, Hin, Cin, K):
    Ho = Hin // 2
    dA = dA[:, :K].reshape(B, Ho, Ho, 9, Cin)
    dHp = np.zeros((B, Hin + 2, Hin + 2, Cin), dtype=dA.dtype)
    for ky in range(3):
        for kx in range(3):
            dHp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Ho:2, :] += dA[:, :, :, ky * 3 + kx, :]
    return dHp[:, 1:-1, 1:-1, :]


def _rounder(rounding):
    """x -> its BF16 value (as float64) in the device's arithmetic; the identity in exact mode."""
    if rounding == "bf16":
        return lambda a: bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)
    return lambda a: np.asarray(a, dtype=np.float64)


def forward(p, X, rounding="bf16"):
    """Outputs (B, 6) and the cache of the backward pass; X (B, 64, 64, 2)."""
    r = _rounder(rounding)
    P = _unpack(np.asarray(p, dtype=np.float64))
    B = X.shape[0]
    H = r(X)
    cache = {"A": [], "H": [H]}
    for l, (Hin, Cin, Cout, K, Kp) in enumerate(CONV):
        A = _im2col(H, Hin, Cin, K, Kp)
        W, b = P[l]
        Z = A @ r(W).T + b
        H = r(np.maximum(Z, 0.0)).reshape(B, Hin // 2, Hin // 2, Cout)
        cache["A"].append(A)
        cache["H"].append(H)
    F = H.reshape(B, 1024)
    W, b = P[4]
    H5 = r(np.maximum(F @ r(W).T + b, 0.0))
    W, b = P[5]
    Y = H5 @ r(W).T + b
    cache["F"], cache["H5"] = F, H5
    return Y[:, :N_OUT], cache


def loss_and_gradients(p, X, T, rounding="bf16"):
    """Mean squared error over B x 6 and its gradient (flat, float64)."""
    r = _rounder(rounding)
    P = _unpack(p)
    B = X.shape[0]
    Y, c = forward(p, X, rounding)
    D = Y - np.asarray(T, dtype=np.float64)
    loss = float(np.mean(D * D))
    dY = np.zeros((B, N_OUTP))
    dY[:, :N_OUT] = 2.0 * D / (B * N_OUT)
    dY = r(dY)
    off, n = layout()
    g = np.zeros(n)

    def put(l, dW, db):
        ow, ob = off[l]
        g[ow:ob] = dW.ravel()
        g[ob:ob + ROWS[l]] = db

    Wq = [r(P[l][0]) for l in range(6)]
    put(5, dY.T @ c["H5"], dY.sum(0))
    dZ = r(dY @ Wq[5] * (c["H5"] > 0))
    put(4, dZ.T @ c["F"], dZ.sum(0))
    dZ = r(dZ @ Wq[4] * (c["F"] > 0))
    for l in range(3, -1, -1):
        Hin, Cin, Cout, K, Kp = CONV[l]
        dZm = dZ.reshape(-1, Cout)
        put(l, dZm.T @ c["A"][l], dZm.sum(0))
        if l == 0:
            break
        dH = _col2im(dZm @ Wq[l], B, Hin, Cin, K)
        dZ = r(dH * (c["H"][l] > 0))
    return loss, g
