"""CPU restatement of the proposal network (test infrastructure only; the product path is the
tensor-core network in 3d-stereo-aldic_b200/csrc/cnn.cu).

The network has no counterpart in the reference (its initial guess is the integer search,
func/funIntegerSearch.m:132-180).  This module restates the device network in numpy so the
device's forward pass, gradients and training step can be checked:

  * rounding="bf16": the device's arithmetic points -- BF16 inputs, BF16 weight copies, BF16
    activations after each ReLU and after the correlation, BF16 output gradient and BF16
    ReLU-masked gradients, with the products accumulated exactly (float64) where the device
    accumulates in FP32;
  * rounding=None: exact float64 math, pinned against central finite differences of the loss
    (tests/test_cnn_oracle.py), which checks the backward formulas themselves.

Architecture (NHWC activations, 3 x 3 convolutions with padding 1):
  input 72 x 72 x 2 centred on the subset: channel 1 the deformed image, channel 0 the
  reference image in the centre 40 x 40
  the reference part R (40 x 40) and the deformed window D (72 x 72) through the same two
      convolutions, conv1 1 -> 32 stride 2, conv2 32 -> 32 stride 2 (R: 10 x 10 x 32, D:
      18 x 18 x 32), of which the inner 8 x 8 and 16 x 16 are kept
  correlation volume C[i, j, d] = sum_c fR[i, j, c] fD[i + 4 + di, j + 4 + dj, c] / 32 over the
      81 offsets d = (di + 4) 9 + (dj + 4), di, dj in -4..4 (+-16 px at stride 4): 8 x 8 x 81
  conv3 81 -> 64 stride 2 (4 x 4), conv4 64 -> 64 stride 1 (4 x 4), FC 1024 -> 128 -> 6.
Layouts follow aldic_net_param_count(): per layer W (rows x cols, row-major) then b; conv K
ordered (ky, kx, channel).
"""
from __future__ import annotations

import numpy as np

ROWS = [32, 32, 64, 64, 128, 16]
COLS = [16, 288, 736, 576, 1024, 128]
FAN_IN = [9, 288, 729, 576, 1024, 128]
N_OUT, N_OUTP = 6, 16
NDISP = 81


def layout():
    """Offsets (w, b) of each layer in the flat parameter vector, and its length."""
    off, o = [], 0
    for r, c in zip(ROWS, COLS):
        off.append((o, o + r * c))
        o += r * c + r
    return off, o


def pad_mask():
    """Boolean mask of the parameter entries that are padding (held at zero)."""
    off, n = layout()
    m = np.zeros(n, dtype=bool)
    for l, (ow, ob) in enumerate(off):
        W = m[ow:ob].reshape(ROWS[l], COLS[l])
        W[:, FAN_IN[l]:] = True
        if l == 5:
            W[N_OUT:, :] = True
            m[ob + N_OUT:ob + ROWS[l]] = True
    return m


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def init_params(seed=0):
    """He-normal weights (std sqrt(2 / fan-in)), zero biases, zero padding (FP32)."""
    off, n = layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    for l, (ow, ob) in enumerate(off):
        W = rng.normal(0.0, np.sqrt(2.0 / FAN_IN[l]), (ROWS[l], COLS[l])).astype(np.float32)
        p[ow:ob] = W.ravel()
    p[pad_mask()] = 0.0
    return p


def _unpack(p):
    off, _ = layout()
    return [(p[ow:ob].reshape(ROWS[l], COLS[l]), p[ob:ob + ROWS[l]]) for l, (ow, ob) in enumerate(off)]


def _im2col(H, stride, Kp):
    """NHWC (B, Hin, Hin, Cin) -> (B * Hout^2, Kp): 3 x 3, pad 1, K = (ky, kx, c)."""
    B, Hin, _, Cin = H.shape
    Ho = (Hin + stride - 1) // stride
    Hp = np.zeros((B, Hin + 2, Hin + 2, Cin), dtype=H.dtype)
    Hp[:, 1:-1, 1:-1, :] = H
    cols = [Hp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Ho:stride, :] for ky in range(3) for kx in range(3)]
    A = np.concatenate(cols, axis=3).reshape(B * Ho * Ho, 9 * Cin)
    if Kp > A.shape[1]:
        A = np.concatenate([A, np.zeros((A.shape[0], Kp - A.shape[1]), dtype=A.dtype)], axis=1)
    return A


def _col2im(dA, B, Hin, Cin, stride):
    Ho = (Hin + stride - 1) // stride
    dA = dA[:, :9 * Cin].reshape(B, Ho, Ho, 9, Cin)
    dHp = np.zeros((B, Hin + 2, Hin + 2, Cin), dtype=dA.dtype)
    for ky in range(3):
        for kx in range(3):
            dHp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Ho:stride, :] += dA[:, :, :, ky * 3 + kx, :]
    return dHp[:, 1:-1, 1:-1, :]


def _rounder(rounding):
    """x -> its BF16 value (as float64) in the device's arithmetic; the identity in exact mode."""
    if rounding == "bf16":
        return lambda a: bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)
    return lambda a: np.asarray(a, dtype=np.float64)


def _shifts():
    return [(di, dj) for di in range(-4, 5) for dj in range(-4, 5)]


def correlation(fR, fD):
    """(B, 8, 8, 81) volume of the 8 x 8 reference features against the 16 x 16 deformed ones."""
    out = np.empty(fR.shape[:3] + (NDISP,))
    for d, (di, dj) in enumerate(_shifts()):
        out[..., d] = np.einsum("bijc,bijc->bij", fR, fD[:, 4 + di:12 + di, 4 + dj:12 + dj, :]) / 32.0
    return out


def correlation_backward(dC, fR, fD):
    dR = np.zeros_like(fR)
    dD = np.zeros_like(fD)
    for d, (di, dj) in enumerate(_shifts()):
        g = dC[..., d:d + 1] / 32.0
        dR += g * fD[:, 4 + di:12 + di, 4 + dj:12 + dj, :]
        dD[:, 4 + di:12 + di, 4 + dj:12 + dj, :] += g * fR
    return dR, dD


def forward(p, X, rounding="bf16"):
    """Outputs (B, 6) and the cache of the backward pass; X (B, 72, 72, 2)."""
    r = _rounder(rounding)
    P = _unpack(np.asarray(p, dtype=np.float64))
    B = X.shape[0]
    X = r(X)
    R, D = X[:, 16:56, 16:56, 0:1], X[:, :, :, 1:2]

    def conv(H, l, stride):
        A = _im2col(H, stride, COLS[l])
        W, b = P[l]
        Ho = (H.shape[1] + stride - 1) // stride
        return A, r(np.maximum(A @ r(W).T + b, 0.0)).reshape(B, Ho, Ho, ROWS[l])

    c = {}
    c["A0"], c["H0"] = conv(R, 0, 2)
    c["A1"], c["H1"] = conv(D, 0, 2)
    c["A2"], c["H2"] = conv(c["H0"], 1, 2)
    c["A3"], c["H3"] = conv(c["H1"], 1, 2)
    c["C"] = r(correlation(c["H2"][:, 1:9, 1:9], c["H3"][:, 1:17, 1:17]))
    c["A4"], c["H4"] = conv(c["C"], 2, 2)
    c["A5"], c["H5"] = conv(c["H4"], 3, 1)
    F = c["H5"].reshape(B, 1024)
    W, b = P[4]
    c["H6"] = r(np.maximum(F @ r(W).T + b, 0.0))
    W, b = P[5]
    Y = c["H6"] @ r(W).T + b
    c["F"] = F
    return Y[:, :N_OUT], c


def loss_and_gradients(p, X, T, rounding="bf16"):
    """Mean squared error over B x 6 and its gradient (flat, float64)."""
    r = _rounder(rounding)
    p = np.asarray(p, dtype=np.float64)
    P = _unpack(p)
    B = X.shape[0]
    Y, c = forward(p, X, rounding)
    Dv = Y - np.asarray(T, dtype=np.float64)
    loss = float(np.mean(Dv * Dv))
    dY = np.zeros((B, N_OUTP))
    dY[:, :N_OUT] = 2.0 * Dv / (B * N_OUT)
    dY = r(dY)
    off, n = layout()
    g = np.zeros(n)

    def put(l, dZ, A):
        ow, ob = off[l]
        g[ow:ob] += (dZ.T @ A).ravel()
        g[ob:ob + ROWS[l]] += dZ.sum(0)

    Wq = [r(P[l][0]) for l in range(6)]
    put(5, dY, c["H6"])
    dZ = r(dY @ Wq[5] * (c["H6"] > 0))
    put(4, dZ, c["F"])
    dZ5 = r(dZ @ Wq[4] * (c["F"] > 0)).reshape(B * 16, 64)
    put(3, dZ5, c["A5"])
    dH4 = _col2im(dZ5 @ Wq[3], B, 4, 64, 1)
    dZ4 = r(dH4 * (c["H4"] > 0)).reshape(B * 16, 64)
    put(2, dZ4, c["A4"])
    dC = _col2im(dZ4 @ Wq[2], B, 8, NDISP, 2)
    dR, dD = correlation_backward(dC, c["H2"][:, 1:9, 1:9], c["H3"][:, 1:17, 1:17])
    dH2, dH3 = np.zeros_like(c["H2"]), np.zeros_like(c["H3"])
    dH2[:, 1:9, 1:9] = dR
    dH3[:, 1:17, 1:17] = dD
    dZ2 = r(dH2 * (c["H2"] > 0)).reshape(-1, 32)
    dZ3 = r(dH3 * (c["H3"] > 0)).reshape(-1, 32)
    put(1, dZ2, c["A2"])
    put(1, dZ3, c["A3"])
    dZ0 = r(_col2im(dZ2 @ Wq[1], B, 20, 32, 2) * (c["H0"] > 0)).reshape(-1, 32)
    dZ1 = r(_col2im(dZ3 @ Wq[1], B, 36, 32, 2) * (c["H1"] > 0)).reshape(-1, 32)
    put(0, dZ0, c["A0"])
    put(0, dZ1, c["A1"])
    return loss, g
