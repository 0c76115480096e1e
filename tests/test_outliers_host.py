"""CPU checks of the integer search's bad-point removal (funRemoveOutliers, Thr0 > 0).

The oracle's restatement is checked against closed forms (method 3 reproduces cubic
surfaces, the median filter's neighbourhood by hand), then the library's per-entry algebra
(outliers.cu, compiled for the host) is compared with the oracle: the method-3 operator
coefficient by coefficient, the CGLS fill against the oracle's least-squares solve, and the
single-precision median test bit for bit.  No GPU is involved.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host", "outliers_check.cu")


def test_inpaint3_reproduces_cubics_and_linear_edges():
    m, n = 30, 25
    R, C = np.meshgrid(np.arange(m, dtype=float), np.arange(n, dtype=float), indexing="ij")
    Z = 0.01 * R ** 3 - 0.02 * C ** 2 * R + 0.5 * C
    A = Z.copy()
    A[10:15, 8:12] = np.nan
    assert np.abs(O.inpaint_nans3(A) - Z).max() < 1e-9
    L = 0.3 * R - 0.2 * C + 1.0  # the edge stencils are exact on linear fields
    A = L.copy()
    A[0, 3] = A[28, 24] = A[1, 1] = np.nan
    assert np.abs(O.inpaint_nans3(A) - L).max() < 1e-12


def test_medfilt2_neighbourhood_by_hand():
    V = np.arange(12.0).reshape(3, 4)
    M = O.medfilt2_skip(V)
    # (0,0): {0, 4, 5}; (0,3): {3, 7, 7 (column repeated)}; (2,3): {11, 11, 11}
    assert M.dtype == np.float32 and M[0, 0] == 4 and M[0, 3] == 7 and M[2, 3] == 11


def test_remove_outliers_oracle_planted():
    R, C = np.meshgrid(np.arange(30.0), np.arange(20.0), indexing="ij")
    u = 3.0 + 0.01 * R
    v = -2.0 + 0.005 * C
    u[5, 5] = 40.0
    v[20, 7] = -60.0
    u[12, 3] = v[12, 3] = np.nan
    u2, v2, bad = O.remove_outliers(u, v)
    assert sorted(bad.tolist()) == sorted([5 + 5 * 30, 20 + 7 * 30])
    assert abs(u2[5, 5] - 3.05) < 1e-9 and abs(v2[20, 7] - (-2.0 + 0.035)) < 1e-9
    assert np.isnan(u2[12, 3]) and np.isnan(v2[12, 3])
    assert np.isfinite(np.delete(u2.ravel(order="F"), 12 + 3 * 30)).all()


TAPS = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1), (-2, 0), (2, 0), (0, -2), (0, 2), (-1, -1), (1, -1), (-1, 1),
        (1, 1)]


def _dense_oracle(m, n):
    """The reference's operator over every entry (its sparse() sums), as a dense matrix."""
    i, j, w = O._del4_rows(m, n, np.arange(m * n))
    ok = (j >= 0) & (j < m * n)  # taps where the reference's sparse() would stop
    D = np.zeros((m * n, m * n))
    np.add.at(D, (i[ok], j[ok]), w[ok])
    return D


def _dense_taps(coef, m, n):
    """The library's per-tap coefficients placed at their linear (column-major) columns;
    on grids of 3 x 3 and more every non-zero tap must also be the in-grid neighbour."""
    D = np.zeros((m * n, m * n))
    for g in range(m * n):
        r, c = g % m, g // m
        for o, (dr, dc) in enumerate(TAPS):
            h = g + dr + dc * m
            if coef[g, o] == 0 or h < 0 or h >= m * n:
                continue
            if m >= 3 and n >= 3:
                assert 0 <= r + dr < m and 0 <= c + dc < n, (g, o)
            D[g, h] += coef[g, o]
    return D


def _run(exe, tmp_path, A, X0, U, V):
    m, n = A.shape
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(np.array([m, n], dtype=np.int32).tobytes())
        for arr in (A, X0, U, V):
            f.write(np.asarray(arr, dtype=np.float64).ravel(order="F").tobytes())
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = open(fout, "rb").read()
    mn = m * n
    coef = np.frombuffer(raw, np.float64, 13 * mn, 0).reshape(mn, 13)
    off = 13 * mn * 8
    fill = np.frombuffer(raw, np.float64, mn, off).reshape((m, n), order="F")
    off += mn * 8
    eq = np.frombuffer(raw, np.int32, mn, off)
    off += mn * 4
    mag = np.frombuffer(raw, np.float32, mn, off).reshape((m, n), order="F")
    return coef, fill, eq, mag, r.stdout


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("outl") / "outliers_check")
    cmd = ["nvcc", "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-o", exe, SRC]
    b = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert b.returncode == 0, b.stderr[-2000:]
    return exe


@pytest.mark.parametrize("m,n", [(1, 6), (2, 5), (3, 3), (4, 4), (5, 7), (9, 12), (6, 2), (7, 1)])
def test_del4_coefficients_match_the_reference_sets(harness, tmp_path, m, n):
    A = np.zeros((m, n))
    coef, _, _, _, _ = _run(harness, tmp_path, A, A, A, A)
    assert np.array_equal(_dense_taps(coef, m, n), _dense_oracle(m, n))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_cgls_fill_matches_the_least_squares_solve(harness, tmp_path, seed):
    rng = np.random.default_rng(seed)
    m, n = 24, 19
    R, C = np.meshgrid(np.arange(m, dtype=float), np.arange(n, dtype=float), indexing="ij")
    Z = np.sin(R / 5.0) + 0.3 * np.cos(C / 3.0) + 0.05 * rng.standard_normal((m, n))
    A = Z.copy()
    A[rng.random((m, n)) < 0.06] = np.nan       # scattered single holes, edges and corners too
    A[8:12, 5:9] = np.nan                      # a 4 x 4 hole
    A[0, 0:3] = np.nan
    X0 = O.inpaint_nans4(A)
    coef, fill, eq, _, out = _run(harness, tmp_path, A, X0, Z, Z)
    ref = O.inpaint_nans3(A)
    assert "met 1" in out, out
    assert np.abs(fill - ref).max() < 1e-8 * max(1.0, np.abs(ref).max())
    # the kept rows: the reference's rows with a non-zero coefficient on a NaN column
    nanf = np.isnan(A.ravel(order="F"))
    want = (_dense_oracle(m, n)[:, nanf] != 0).any(1).astype(np.int32)
    assert np.array_equal(eq, want)


def test_median_test_is_bit_exact(harness, tmp_path):
    rng = np.random.default_rng(5)
    m, n = 31, 27
    U = 3.0 + 0.01 * rng.standard_normal((m, n)) + np.round(rng.random((m, n)) * 3) * 1e-3
    V = -2.0 + 0.02 * rng.standard_normal((m, n))
    U[rng.random((m, n)) < 0.03] += 40.0
    V[rng.random((m, n)) < 0.03] -= 25.0
    A = np.zeros((m, n))
    _, _, _, mag, _ = _run(harness, tmp_path, A, A, U, V)
    med_u = O.medfilt2_skip(U)
    fu = (U.astype(np.float32) - med_u).astype(np.float32)
    fv = (V.astype(np.float32) - O.medfilt2_skip(V)).astype(np.float32)
    nu = np.abs(fu / (O.medfilt2_skip(np.abs(fu)) + np.float32(0.1)))
    nv = np.abs(fv / (O.medfilt2_skip(np.abs(fv)) + np.float32(0.1)))
    want = np.sqrt(nu * nu + nv * nv).astype(np.float32)
    assert np.array_equal(mag.view(np.uint32), want.view(np.uint32))
    assert (mag > 100).sum() > 0
