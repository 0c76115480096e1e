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


def test_init_index1_removes_outliers_and_index0_keeps_them():
    rng = np.random.default_rng(1)
    y, x = np.mgrid[0:20, 0:25]
    u = 0.02 * x + 0.01 * y + rng.normal(0, 0.01, x.shape)
    v = -0.03 * x + rng.normal(0, 0.01, x.shape)
    u[5, 7] += 3.0
    v[12, 15] -= 2.0
    u[3, 3] = np.nan
    U1 = O.init_u0(u, v, index=1)
    U0 = O.init_u0(u, v, index=0)
    u1, v1 = U1[0::2].reshape(20, 25), U1[1::2].reshape(20, 25)
    assert abs(u1[5, 7] - (0.02 * 7 + 0.01 * 5)) < 0.05
    assert abs(v1[12, 15] - (-0.03 * 15)) < 0.05
    assert abs(U0[0::2].reshape(20, 25)[5, 7] - u[5, 7]) < 1e-12
    assert np.isfinite(U1).all()


def test_spring_pass_statistics_follow_matlab():
    # std over the neighbours is the N-1 sample deviation, NaN entries omitted
    assert abs(O._std8([1.0, 2.0, 3.0, 4.0]) - np.std([1, 2, 3, 4], ddof=1)) < 1e-15
    assert abs(O._std8([1.0, np.nan, 3.0]) - np.std([1, 3], ddof=1)) < 1e-15
    assert O._std8([5.0]) == 0.0 and np.isnan(O._std8([np.nan]))


def test_undistort_is_the_inverse_of_the_lens_model():
    K = np.array([[4000.0, 0.5, 1024.5], [0, 4010.0, 1000.2], [0, 0, 1]])
    rng = np.random.default_rng(0)
    P = rng.uniform(1, 2048, (500, 2))
    for rad, tan in (([-0.12, 0.05, -0.01], [1e-3, -5e-4]), ([0.08, -0.02], None)):
        U = O.undistort_points(P, K, rad, tan)
        assert np.abs(O.distort_points(U, K, rad, tan) - P).max() < 1e-9
    # zero distortion: the identity (through K and back)
    assert np.abs(O.undistort_points(P, K, [0.0, 0.0]) - P).max() < 1e-9
    Q = P.copy()
    Q[3, 1] = np.nan
    assert np.isnan(O.undistort_points(Q, K, [0.1, 0.0])[3]).all()
