"""CPU checks of the proposal network's restatement (oracle/cnn_oracle.py), the checker of
the device network: its backward pass in exact float64 against central finite differences
of its loss, and its BF16 rounding."""
import numpy as np

import cnn_oracle as CO


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-3], dtype=np.float32)
    got = CO.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1); 1 + 3 * 2^-8 rounds up
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == np.float32(1.0 + 2 ** -6) and got[3] == 1.0
    assert got[4] == -2.5
    assert abs(got[5] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_exact_gradients_match_finite_differences():
    # per layer, weights and biases: the directional derivative along a random unit direction
    # (padding entries held at zero) against a central difference of the loss (small enough a
    # step that no ReLU changes side)
    rng = np.random.default_rng(0)
    p = CO.init_params(3).astype(np.float64)
    p[~CO.pad_mask()] += rng.normal(scale=0.02, size=int((~CO.pad_mask()).sum()))  # nonzero biases
    X = rng.normal(size=(2, 72, 72, 2))
    T = rng.normal(scale=0.3, size=(2, 6))
    loss, g = CO.loss_and_gradients(p, X, T, rounding=None)
    assert np.isfinite(loss) and np.abs(g).max() > 0
    off, n = CO.layout()
    pad = CO.pad_mask()
    eps = 1e-6
    for l, (ow, ob) in enumerate(off):
        for a, b in ((ow, ob), (ob, ob + CO.ROWS[l])):
            d = np.zeros(n)
            d[a:b] = rng.normal(size=b - a)
            d[pad] = 0.0
            d /= np.linalg.norm(d)
            lp, _ = CO.loss_and_gradients(p + eps * d, X, T, rounding=None)
            lm, _ = CO.loss_and_gradients(p - eps * d, X, T, rounding=None)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g @ d) <= 1e-6 * max(1e-3, abs(fd)), (l, fd, g @ d)
    # padding entries get no gradient
    assert np.all(g[pad] == 0.0)


def test_correlation_volume_and_its_gradient():
    # the volume against a direct loop, and its backward pass as the adjoint of the forward
    rng = np.random.default_rng(1)
    fR = rng.normal(size=(2, 8, 8, 32))
    fD = rng.normal(size=(2, 16, 16, 32))
    C = CO.correlation(fR, fD)
    b, i, j, di, dj = 1, 3, 5, -4, 2
    want = fR[b, i, j] @ fD[b, i + 4 + di, j + 4 + dj] / 32.0
    assert abs(C[b, i, j, (di + 4) * 9 + (dj + 4)] - want) < 1e-12
    dC = rng.normal(size=C.shape)
    dR, dD = CO.correlation_backward(dC, fR, fD)
    eR, eD = rng.normal(size=fR.shape), rng.normal(size=fD.shape)
    # linear in each argument: <dC, C(eR, fD)> = <dR, eR>, <dC, C(fR, eD)> = <dD, eD>
    assert abs(np.sum(dC * CO.correlation(eR, fD)) - np.sum(dR * eR)) < 1e-9
    assert abs(np.sum(dC * CO.correlation(fR, eD)) - np.sum(dD * eD)) < 1e-9
