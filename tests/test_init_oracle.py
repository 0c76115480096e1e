"""CPU checks of the oracle's Init / inpaint_nans(., 4) restatement: the spring system's
solution is the discrete harmonic interpolant (every NaN entry the mean of its in-grid
4-neighbours), which a dense solve of those equations gives independently."""
import numpy as np

import oracle as O


def _harmonic(A):
    m, n = A.shape
    nan = [tuple(p) for p in np.argwhere(np.isnan(A))]
    idx = {p: i for i, p in enumerate(nan)}
    M = np.zeros((len(nan), len(nan)))
    b = np.zeros(len(nan))
    for i, (r, c) in enumerate(nan):
        for dr, dc in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            rr, cc = r + dr, c + dc
            if 0 <= rr < m and 0 <= cc < n:
                M[i, i] += 1
                if (rr, cc) in idx:
                    M[i, idx[(rr, cc)]] -= 1
                else:
                    b[i] += A[rr, cc]
    out = A.copy()
    x = np.linalg.solve(M, b)
    for i, p in enumerate(nan):
        out[p] = x[i]
    return out


def test_inpaint_nans4_is_the_harmonic_fill():
    rng = np.random.default_rng(3)
    A = rng.normal(size=(13, 17))
    A[rng.random(A.shape) < 0.15] = np.nan   # scattered
    A[4:8, 5:10] = np.nan                     # a block hole
    A[0, :6] = np.nan                         # on the border
    A[:, -1] = np.nan                         # a whole edge column
    B = O.inpaint_nans4(A)
    assert np.isfinite(B).all()
    assert np.array_equal(B[np.isfinite(A)], A[np.isfinite(A)])
    assert np.abs(B - _harmonic(A)).max() < 1e-12


def test_inpaint_reproduces_linear_fields_and_init_order():
    # a linear field is harmonic: holes in it are filled exactly
    y, x = np.mgrid[0:11, 0:14]
    A = 0.3 * x - 0.7 * y + 2.0
    H = A.copy()
    H[3:7, 4:9] = np.nan
    assert np.abs(O.inpaint_nans4(H) - A).max() < 1e-12
    # Init interleaves the transposed grids: XList (the second axis of u) fastest
    u = np.arange(12.0).reshape(3, 4)         # ny = 3, nx = 4
    v = -u
    U0 = O.init_u0(u, v)
    assert np.array_equal(U0[0::2], u.T.ravel(order="F"))
    assert np.array_equal(U0[1::2], v.T.ravel(order="F"))
    assert U0[0] == u[0, 0] and U0[2] == u[0, 1]
