"""CPU checks of the natural-neighbour fill (MATLAB scatteredInterpolant 'natural').

The library's Sibson coordinates (Delaunay-cavity candidates, exact half-plane clipping)
are compared with the oracle's brute-force restatement of the definition (every point clips
every cell), and with Sibson's properties: partition of unity, linear precision inside the
hull, the centroid property, the edge-linear limit on hull edges, 'nearest' / 'none'
outside.  Then the drivers' fills on meshes with NaN holes.  No GPU is involved.
"""
import numpy as np
import pytest

import oracle as O
from aldic_b200.fill import NaturalNeighbor, fill_nans_natural, fill_quadtree


def _lin(X):
    return 2.0 + 0.3 * X[..., 0] - 0.7 * X[..., 1]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sibson_matches_the_bruteforce_definition(seed):
    rng = np.random.default_rng(seed)
    P = rng.random((60, 2)) * 10
    nn = NaturalNeighbor(P)
    for q in rng.random((25, 2)) * 8 + 1:
        idx, w = nn.weights(q)
        wb, bounded = O.sibson_bruteforce(P, q)
        if idx is None:
            assert not bounded
            continue
        full = np.zeros(len(P))
        full[idx] = w
        assert bounded and np.abs(full - wb).max() < 1e-10
        assert abs(w.sum() - 1) < 1e-12 and np.abs(w @ P[idx] - q).max() < 1e-9


def test_grid_with_holes_linear_precision_and_hull():
    pts = np.array([(x, y) for x in range(12) for y in range(10)], dtype=float) * 8 + 10
    hole = ((pts[:, 0] - 50) ** 2 + (pts[:, 1] - 46) ** 2) < 20 ** 2
    hole |= (pts[:, 0] == 10) & (pts[:, 1] == 42)   # a border node (on the hull edge)
    P, Q = pts[~hole], pts[hole]
    nn = NaturalNeighbor(P, "nearest")
    got = nn(Q, _lin(P))
    assert np.abs(got - _lin(Q)).max() < 1e-9      # interior and hull-edge queries alike
    for q in Q[:6]:
        idx, w = nn.weights(q)
        if idx is not None:
            wb, _ = O.sibson_bruteforce(P, q)
            full = np.zeros(len(P))
            full[idx] = w
            assert np.abs(full - wb).max() < 1e-10
    far = np.array([[500.0, 500.0]])
    assert np.array_equal(nn(far, _lin(P)), _lin(P[[np.argmin(((P - far) ** 2).sum(1))]]))
    assert np.isnan(NaturalNeighbor(P, "none")(far, _lin(P))).all()


def test_fill_nans_natural_and_quadtree_regions():
    pts = np.array([(x, y) for x in range(14) for y in range(14)], dtype=float) * 8 + 10
    n = len(pts)
    U = np.stack([_lin(pts), 0.5 * _lin(pts)], 1)
    bad = np.zeros(n, bool)
    bad[[20, 21, 35, 100, 101, 150]] = True
    Ub = U.copy()
    Ub[bad] = np.nan
    assert np.abs(fill_nans_natural(pts, Ub) - U).max() < 1e-9
    # two mask regions split by a vertical gap: each region's NaN nodes come from its own nodes
    mask = np.ones((140, 140))
    mask[59:63, :] = 0  # pixels 60-63: between the node columns at 58 and 66
    left = pts[:, 0] < 60
    Uq = U.copy()
    Uq[left, 0] += 100.0                      # the left region lives on another level
    Uqb = Uq.copy()
    Uqb[bad] = np.nan
    out = fill_quadtree(Uqb.ravel(), pts, mask).reshape(-1, 2)
    assert np.abs(out - Uq).max() < 1e-9      # no blending across the gap


def test_native_weights_match_the_python_construction():
    """The library's host code (aldic_sibson_weights) against the Python construction and
    the brute-force definition, on random points and on a grid with a large hole."""
    rng = np.random.default_rng(9)
    cases = [rng.random((120, 2)) * 10]
    pts = np.array([(x, y) for x in range(30) for y in range(30)], dtype=float) * 8 + 10
    hole = ((pts[:, 0] - 130) ** 2 + (pts[:, 1] - 120) ** 2) < 60 ** 2
    cases.append(pts[~hole])
    queries = [rng.random((60, 2)) * 9 + 0.5, pts[hole]]
    for P, Q in zip(cases, queries):
        nn = NaturalNeighbor(P)
        idx, w, cnt = nn.native_weights(Q)
        assert (cnt > 0).mean() > 0.8
        for m, q in enumerate(Q):
            if cnt[m] <= 0:
                continue
            a = np.zeros(len(P))
            a[idx[m, :cnt[m]]] = w[m, :cnt[m]]
            i2, w2 = nn.weights(q)
            b = np.zeros(len(P))
            b[i2] = w2
            assert np.abs(a - b).max() < 1e-12
        for m in range(0, len(Q), 20):
            if cnt[m] > 0 and len(P) <= 150:  # the definition by brute force: small sets only
                a = np.zeros(len(P))
                a[idx[m, :cnt[m]]] = w[m, :cnt[m]]
                wb, _ = O.sibson_bruteforce(P, Q[m])
                assert np.abs(a - wb).max() < 1e-10


def _gridfit_dense(xn, yn, data, smoothness=1.0):
    """The springs fit by a separate construction: one row per finite node value, one per
    spring between grid neighbours (right, up, both diagonals), dense least squares."""
    nx, ny = len(xn), len(yn)
    idx = lambda i, j: j + ny * i  # noqa: E731  (column-major node number, as MATLAB's grid)
    A, z = [], []
    for i in range(nx):
        for j in range(ny):
            if np.isfinite(data[j, i]):
                r = np.zeros(nx * ny)
                r[idx(i, j)] = 1.0
                A.append(r)
                z.append(data[j, i])
    A = np.array(A)
    sx, sy = np.mean(np.diff(xn)), np.mean(np.diff(yn))
    reg = []
    for i in range(nx):
        for j in range(ny):
            for di, dj in ((0, 1), (1, 0), (1, 1), (1, -1)):
                i2, j2 = i + di, j + dj
                if not (0 <= i2 < nx and 0 <= j2 < ny):
                    continue
                h = np.hypot((xn[i2] - xn[i]) / sx * (di != 0), (yn[j2] - yn[j]) / sy * (dj != 0))
                r = np.zeros(nx * ny)
                r[idx(i, j)], r[idx(i2, j2)] = -1.0 / h, 1.0 / h
                reg.append(r)
    R = np.array(reg)
    lam = smoothness * np.abs(A).sum(0).max() / np.abs(R).sum(0).max()
    S = np.vstack([A, lam * R])
    sol = np.linalg.lstsq(S, np.concatenate([z, np.zeros(len(R))]), rcond=None)[0]
    return sol.reshape((nx, ny)).T


def test_gridfit_springs_matches_a_separate_construction():
    from aldic_b200.fill import gridfit_springs

    rng = np.random.default_rng(4)
    xn = np.array([10.0, 18.0, 26.0, 34.0, 42.0, 50.0])
    yn = np.array([5.0, 13.0, 21.0, 29.0, 37.0])
    X, Y = np.meshgrid(xn, yn)                     # ny x nx
    data = 0.3 * X - 0.1 * Y + np.sin(X / 7.0) + 0.05 * rng.standard_normal(X.shape)
    data[2, 3] = data[0, 0] = data[4, 5] = np.nan  # the fit covers them
    got = gridfit_springs(X.ravel(), Y.ravel(), data.ravel(), xn, yn)
    want = _gridfit_dense(xn, yn, data)
    assert got.shape == (5, 6) and np.abs(got - want).max() < 1e-10
    # the 'triangle' rule off the nodes: a cell centre is the mean of the cell's diagonal
    # corners, so a plane sampled there, with vanishing smoothing, comes back exactly
    cx = (X[:-1, :-1] + X[1:, 1:]).ravel() / 2
    cy = (Y[:-1, :-1] + Y[1:, 1:]).ravel() / 2
    plane = lambda a, b: 1.0 + 0.2 * a - 0.3 * b  # noqa: E731
    pts_x = np.concatenate([X.ravel(), cx])
    pts_y = np.concatenate([Y.ravel(), cy])
    zg = gridfit_springs(pts_x, pts_y, plane(pts_x, pts_y), xn, yn, smoothness=1e-9)
    assert np.abs(zg - plane(X, Y)).max() < 1e-6
