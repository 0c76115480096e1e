"""CPU checks of the ALDIC loop's optional displacement smoothing (funSmoothDispQuadtree):
the regularised lattice fit against a separate dense construction of the same least-squares
system, the NaN-aware Gaussian filter against explicit sums, and the whole smoothing on
fields with a known answer.  No GPU is involved."""
import numpy as np

from aldic_b200.smooth import funSmoothDispQuadtree, gaussian_kernel, nanconv_edge, regularize_2d


def _regularize_dense(xy, z, xn, yn, s):
    n1, n2, n = len(xn), len(yn), len(z)
    rows = []
    for (x, y) in xy:  # bilinear weights of the point's cell
        i = min(max(np.searchsorted(xn, x, side="right") - 1, 0), n1 - 2)
        j = min(max(np.searchsorted(yn, y, side="right") - 1, 0), n2 - 2)
        fx, fy = (x - xn[i]) / (xn[i + 1] - xn[i]), (y - yn[j]) / (yn[j + 1] - yn[j])
        r = np.zeros(n1 * n2)
        for a, b, w in ((0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)), (0, 1, (1 - fx) * fy), (1, 1, fx * fy)):
            r[(i + a) + n1 * (j + b)] += w
        rows.append(r)
    reg = []
    for d, g in ((0, xn), (1, yn)):
        m = (len(g) - 2) * (n2 if d == 0 else n1)
        scale = s * np.sqrt(n / m) * (g[-1] - g[0]) ** 2
        for a in range(n1 if d == 1 else n1 - 2):
            for b in range(n2 if d == 0 else n2 - 2):
                k = a if d == 0 else b
                x1, x2, x3 = g[k], g[k + 1], g[k + 2]
                ws = 2 / ((x1 - x3) * (x1 - x2)), 2 / ((x2 - x1) * (x2 - x3)), 2 / ((x3 - x1) * (x3 - x2))
                r = np.zeros(n1 * n2)
                for t, w in enumerate(ws):
                    ia, ib = (a + t, b) if d == 0 else (a, b + t)
                    r[ia + n1 * ib] = scale * w
                reg.append(r)
    S = np.vstack([np.array(rows), np.array(reg)])
    sol = np.linalg.lstsq(S, np.concatenate([z, np.zeros(len(reg))]), rcond=None)[0]
    return sol.reshape((n1, n2), order="F")


def test_regularize_2d_matches_a_separate_construction_and_keeps_planes():
    rng = np.random.default_rng(3)
    xn = np.array([0.0, 4.0, 8.0, 12.0, 16.0, 20.0])
    yn = np.array([0.0, 4.0, 8.0, 12.0, 16.0])
    xy = np.stack([rng.uniform(0, 20, 70), rng.uniform(0, 16, 70)], 1)
    z = np.sin(xy[:, 0] / 5) + 0.2 * xy[:, 1] + 0.05 * rng.standard_normal(70)
    got = regularize_2d(xy, z, xn, yn, 5e-4)
    assert np.abs(got - _regularize_dense(xy, z, xn, yn, 5e-4)).max() < 1e-9
    plane = 1.0 + 0.3 * xy[:, 0] - 0.2 * xy[:, 1]     # second differences vanish: exact
    g2 = regularize_2d(xy, plane, xn, yn, 0.1)
    X, Y = np.meshgrid(xn, yn, indexing="ij")
    assert np.abs(g2 - (1.0 + 0.3 * X - 0.2 * Y)).max() < 1e-9


def test_nanconv_edge_explicit_sums():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((7, 6))
    a[2, 3] = a[0, 0] = np.nan
    k = gaussian_kernel(3, 0.5)
    assert abs(k.sum() - 1) < 1e-15 and k[1, 1] == k.max()
    c = nanconv_edge(a, k)
    for i in range(7):
        for j in range(6):
            if np.isnan(a[i, j]):
                assert np.isnan(c[i, j])
                continue
            num = den = 0.0
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    ii, jj = i + di, j + dj
                    if 0 <= ii < 7 and 0 <= jj < 6 and np.isfinite(a[ii, jj]):
                        num += k[1 + di, 1 + dj] * a[ii, jj]
                        den += k[1 + di, 1 + dj]
            assert abs(c[i, j] - num / den) < 1e-13


def test_smoothing_keeps_planes_inside_and_lowers_noise():
    xs = np.arange(10.0, 91.0, 4.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    C = np.stack([X.ravel(), Y.ravel()], 1)
    U = np.stack([0.5 + 0.01 * C[:, 0], -0.3 + 0.02 * C[:, 1]], 1).ravel()
    mesh = {"coordinatesFEM": C, "elementMinSize": 4}
    para = {"DispFilterStd": 0, "DispFilterSize": 0, "DispSmoothness": 5e-4}
    S = funSmoothDispQuadtree(U, mesh, para)
    inner = (C[:, 0] > 14) & (C[:, 0] < 86) & (C[:, 1] > 14) & (C[:, 1] < 86)
    # the filter's edge correction bends a plane at the border; the second pass's global fit
    # carries a trace of that inward
    assert np.abs(S - U).reshape(-1, 2)[inner].max() < 1e-3
    rng = np.random.default_rng(2)
    noisy = U + 0.05 * rng.standard_normal(U.size)
    S2 = funSmoothDispQuadtree(noisy, mesh, para)
    assert np.std((S2 - U).reshape(-1, 2)[inner]) < 0.5 * np.std((noisy - U).reshape(-1, 2)[inner])
