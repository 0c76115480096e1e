"""CPU tests of the FP64 oracle: pinned against the reference's own MEX output (golden
vectors) and against independent restatements of the published toolbox definitions."""
import os

import numpy as np
import pytest

import oracle as O
from aldic_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "interp_golden.npz")


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build()


def test_interp_matches_reference_golden():
    g = np.load(GOLDEN)
    for name in ("speckle", "ramp", "normalised"):
        F, X, Y, Z = g[f"{name}_F"], g[f"{name}_X"], g[f"{name}_Y"], g[f"{name}_Z"]
        z = O.interp(F, X, Y)
        scale = np.abs(Z).max()
        assert np.max(np.abs(z - Z)) <= 1e-13 * max(scale, 1.0), name


def test_interp_ramp_bias_is_reference_behaviour():
    # the truncated prefilter does not reproduce ramps exactly (59.2567 vs 59.25 style bias)
    g = np.load(GOLDEN)
    F, X, Y, Z = g["ramp_F"], g["ramp_X"], g["ramp_Y"], g["ramp_Z"]
    exact = 1.5 * Y + 7.0
    assert np.max(np.abs(Z - exact)) > 1e-4
    assert np.max(np.abs(Z - exact)) < 0.05


def test_interp_integer_points_return_samples():
    rng = np.random.default_rng(3)
    F = rng.normal(size=(20, 17))
    i = rng.integers(4, 16, 50)
    j = rng.integers(4, 13, 50)
    z = O.interp(F, (j + 1).astype(float), (i + 1).astype(float))
    assert np.allclose(z, F[i, j], atol=1e-12)


def test_normalize_matches_numpy():
    rng = np.random.default_rng(1)
    img = rng.integers(0, 255, (40, 30)).astype(float)
    out, ms = O.normalize(img, [3, 35], [2, 28])
    roi = img[2:35, 1:28]
    assert np.isclose(ms[0], roi.mean()) and np.isclose(ms[1], roi.std(ddof=1))
    assert np.allclose(out, (img - roi.mean()) / roi.std(ddof=1))


def test_gradient_matches_convolution():
    rng = np.random.default_rng(2)
    img = rng.normal(size=(30, 26))
    mask = (rng.uniform(size=img.shape) > 0.2).astype(float)
    gx, gy = O.gradient(img, mask)
    h = np.array([-1 / 60, 3 / 20, -3 / 4, 0, 3 / 4, -3 / 20, 1 / 60])
    ex = np.zeros((24, 20))
    ey = np.zeros((24, 20))
    for k in range(7):
        ex += h[k] * img[k:k + 24, 3:23]
        ey += h[k] * img[3:27, k:k + 20]
    assert np.allclose(gx, ex * mask[3:27, 3:23], atol=1e-12)
    assert np.allclose(gy, ey * mask[3:27, 3:23], atol=1e-12)


def _ncc_bruteforce(T, A):
    m, n = T.shape
    ma, na = A.shape
    P = np.zeros((ma + 2 * (m - 1), na + 2 * (n - 1)))
    P[m - 1:m - 1 + ma, n - 1:n - 1 + na] = A
    out = np.zeros((ma + m - 1, na + n - 1))
    Tc = T - T.mean()
    dT = np.sqrt((Tc ** 2).sum())
    dens = np.zeros_like(out)
    nums = np.zeros_like(out)
    for r in range(out.shape[0]):
        for c in range(out.shape[1]):
            W = P[r:r + m, c:c + n]
            nums[r, c] = (Tc * W).sum()
            dens[r, c] = dT * np.sqrt(max((W ** 2).sum() - W.sum() ** 2 / (m * n), 0))
    tol = np.sqrt(np.spacing(dens.max()))
    nz = dens > tol
    out[nz] = nums[nz] / dens[nz]
    out[np.abs(out) - 1 > np.sqrt(np.spacing(1.0))] = 0
    return out


def test_normxcorr2_matches_definition():
    rng = np.random.default_rng(4)
    T = rng.normal(size=(5, 4))
    A = rng.normal(size=(9, 8))
    A[0:3, 0:3] = 0.7  # a flat patch: zero-variance windows give 0
    got = O.normxcorr2(T, A)
    want = _ncc_bruteforce(T, A)
    assert np.allclose(got, want, atol=1e-12)


def test_normxcorr2_rejects_constant_template():
    with pytest.raises(ValueError):
        O.normxcorr2(np.ones((3, 3)), np.random.default_rng(0).normal(size=(6, 6)))


def test_findpeak_matches_lstsq_fit():
    rng = np.random.default_rng(5)
    xs = np.array([-1, -1, -1, 0, 0, 0, 1, 1, 1.0])
    ys = np.array([-1, 0, 1, -1, 0, 1, -1, 0, 1.0])
    X = np.stack([np.ones(9), xs, ys, xs * ys, xs ** 2, ys ** 2], 1)
    for _ in range(200):
        x0, y0 = rng.uniform(-0.45, 0.45, 2)
        f = np.zeros((7, 6))
        rr, cc = np.meshgrid(np.arange(7), np.arange(6), indexing="ij")
        f = 1 - 0.3 * ((cc - 3 - x0) ** 2 + (rr - 3 - y0) ** 2) + 0.01 * rng.normal(size=f.shape)
        xp, yp, mf = O.findpeak(f)
        r, c = np.unravel_index(np.argmax(f.ravel(order="F")), f.shape, order="F")
        u = f[r - 1:r + 2, c - 1:c + 2].ravel(order="F")
        A = np.linalg.lstsq(X, u, rcond=None)[0]
        den = A[3] ** 2 - 4 * A[4] * A[5]
        xo = (-A[2] * A[3] + 2 * A[5] * A[1]) / den
        yo = -1 / den * (A[3] * A[1] - 2 * A[4] * A[2])
        if abs(xo) > 1 or abs(yo) > 1:
            continue
        # MATLAB round: half away from zero
        rxo = np.sign(xo) * np.floor(abs(1000 * xo) + 0.5) / 1000
        ryo = np.sign(yo) * np.floor(abs(1000 * yo) + 0.5) / 1000
        assert abs(xp - (c + 1 + rxo)) < 1e-9 and abs(yp - (r + 1 + ryo)) < 1e-9


def test_findpeak_edge_returns_integer_peak():
    f = np.zeros((5, 5))
    f[0, 2] = 1.0
    xp, yp, mf = O.findpeak(f)
    assert (xp, yp, mf) == (3.0, 1.0, 1.0)


def test_bwselect_matches_label():
    from scipy import ndimage

    rng = np.random.default_rng(6)
    for conn in (4, 8):
        for _ in range(20):
            bw = (rng.uniform(size=(21, 17)) > 0.45).astype(np.uint8)
            r, c = rng.integers(0, 21), rng.integers(0, 17)
            got = O.bwselect(bw, r, c, conn)
            st = ndimage.generate_binary_structure(2, 1 if conn == 4 else 2)
            lab, _ = ndimage.label(bw, structure=st)
            want = (lab == lab[r, c]) & (bw > 0) if bw[r, c] else np.zeros_like(bw, dtype=bool)
            assert np.array_equal(got.astype(bool), want)


@pytest.fixture(scope="module")
def affine_small():
    sc = synth.temporal_affine(M=192, N=176, n_speckles=600)
    M, N = sc.ref.shape
    f, _ = O.normalize(sc.ref.astype(float), [1, M], [1, N])
    g, _ = O.normalize(sc.deff.astype(float), [1, M], [1, N])
    gx, gy = O.gradient(f)
    return sc, f, g, gx, gy


def test_integer_search_recovers_shift(affine_small):
    sc, f, g, gx, gy = affine_small
    r = O.integer_search(f, g, [8, 8], [1, f.shape[0]], [1, f.shape[1]], 24, 16)
    tu, tv = sc.disp(r["x"], r["y"])
    ok = np.isfinite(r["u"])
    assert ok.all()
    # the first grid row/column has its search clamped at the image edge (L = ii - 1)
    inner = (r["x"] > 20) & (r["y"] > 20)
    assert np.max(np.abs(r["u"] - tu)[inner]) < 0.7 and np.max(np.abs(r["v"] - tv)[inner]) < 0.7
    edge = r["y"] < 20
    assert np.all(r["v"][edge] >= -1.0)  # clamped: cannot reach the true -1.8 px
    assert np.all(np.abs(r["u"] * 1000 - np.round(r["u"] * 1000)) < 1e-6)  # 1e-3 px rounding


@pytest.mark.parametrize("variant", [0, 1])
def test_icgn_recovers_affine(affine_small, variant):
    sc, f, g, gx, gy = affine_small
    xs = np.arange(30, 160, 13.0)
    ys = np.arange(30, 150, 13.0)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    fr = O.Frame(f, g, None if variant == 0 else np.ones_like(f), gx, gy)
    res = O.local_icgn(fr, coords, U0, 30, 1e-3, variant=variant)
    assert np.all((res["conv"] > 0) & (res["conv"] < 100))
    assert np.max(np.abs(res["U"][0::2] - tu)) < 0.05 and np.max(np.abs(res["U"][1::2] - tv)) < 0.05
    assert np.max(np.abs(res["F"][0::4] - sc.dudx)) < 0.01


def test_icgn_status_codes(affine_small):
    sc, f, g, gx, gy = affine_small
    M, N = f.shape
    mask = np.ones_like(f)
    mask[100:160, 100:160] = 0  # hole
    gxm, gym = O.gradient(f, mask)
    fr = O.Frame(f, g, mask, gxm, gym)
    coords = np.array([[10.0, 90.0],     # window leaves the gradient array -> -1
                       [130.0, 130.0],   # fully masked -> 102
                       [60.0, 60.0],     # clean
                       [100.0, 90.0]])   # partly masked -> enlarged window
    U0 = np.tile([3.0, -2.0], 4)
    res = O.local_icgn(fr, coords, U0, 20, 1e-3, variant=1)
    assert res["conv"][0] == -1 and np.isnan(res["U"][0])
    assert res["conv"][1] == 102 and res["U"][2] == 3.0 and res["F"][4] == 0.0
    assert 0 < res["conv"][2] < 100
    assert res["markHole"][1] == 1 and res["markHole"][2] == 0


def test_subpb1_quadtree_moves_toward_dual_target(affine_small):
    sc, f, g, gx, gy = affine_small
    coords = np.array([[60.0, 70.0], [90.0, 100.0]])
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    UOld = np.stack([tu, tv], 1).ravel() + 0.3
    FOld = np.tile([sc.dudx, 0, 0, sc.dvdy], 2)
    fr = O.Frame(f, g, np.ones_like(f), gx, gy)
    r = O.subpb1(fr, coords, UOld, FOld, np.zeros(4), 1e-3, 1e-3, winsize_list=np.full((2, 2), 24), variant=1)
    assert np.all((r["conv"] > 0) & (r["conv"] < 100))
    assert np.max(np.abs(r["U"][0::2] - tu)) < 0.1


def test_triangulation_recovers_plane():
    st = synth.stereo_pair(size=192, f=400.0)
    rng = np.random.default_rng(7)
    pts = rng.uniform(40, 150, (50, 2))
    tr = synth.stereo_truth(st, pts)
    pairs = np.hstack([pts, tr["right0"]])
    xyz, err = O.triangulate(pairs, st.KL, st.KR, st.R_rl, st.T_rl)
    want = synth.to_left_camera_frame(st, tr["xyz0"])
    assert np.max(np.abs(xyz - want)) < 1e-6 * np.abs(want).max()
    assert np.max(err) < 1e-6
    pairs[3, 2] = np.nan
    xyz, err = O.triangulate(pairs, st.KL, st.KR, st.R_rl, st.T_rl)
    assert np.all(np.isnan(xyz[3])) and np.isnan(err[3])
