"""Host-side driver logic mirrored from the reference (no GPU): bad-point rules of the
local solvers and Subpb1, the search grid, and argument validation of the host API."""
import numpy as np
import pytest

from aldic_b200 import api


def test_bad_points_quadtree_rules():
    # LocalICGNQuadtree.m:169-192: codes < 0 or > 99 are bad; 102 does not count in the
    # bad number; iterations > max(mu + sigma, 6) are bad too
    conv = np.array([3, 4, 5, 4, 3, 30, -1, 101, 102, 103, 4, 5, 6, 7])
    bad, num = api.bad_points_local(conv, rule="quadtree")
    good = conv[(conv >= 0) & (conv <= 99)]
    thr = max(good.mean() + good.std(ddof=1), 6)
    want = np.nonzero((conv < 0) | (conv > 99) | (conv > thr))[0]
    assert np.array_equal(bad, want)
    assert num == 4 - 1  # -1, 101, 102, 103 minus the 102


def test_bad_points_uniform_rule():
    conv = np.array([3, 3, 4, 10, 3, -1])
    bad, num = api.bad_points_local(conv, rule="uniform")
    g = conv[(conv >= 0) & (conv <= 99)]
    thr = g.mean() + 0.15 * g.std(ddof=1)
    assert np.array_equal(bad, np.nonzero((conv < 0) | (conv > 99) | (conv > thr))[0])


def test_bad_points_subpb1_rule():
    conv = np.array([2, 3, 2, 12, 0, 101])
    bad, num = api.bad_points_subpb1(conv)
    g = conv[(conv >= 0) & (conv <= 99)]
    thr = max(g.mean() + 0.25 * g.std(ddof=1), 10)
    assert np.array_equal(bad, np.nonzero((conv < 0) | (conv > 99) | (conv > thr))[0])
    assert num == 1


def test_few_good_points_skip_the_iteration_filter():
    conv = np.array([3, 101, -1])
    bad, _ = api.bad_points_local(conv, rule="quadtree")
    assert list(bad) == [1, 2]


def test_count_and_shape_validation():
    with pytest.raises(api.AldicError):
        api._count(np.zeros((5, 3)), 2)
    assert api._count(np.zeros((5, 2)), 2) == 5
    assert api._img_shape(np.zeros((4, 7)), None) == (4, 7)


def test_funintegersearch_rejects_seed_mode():
    with pytest.raises(api.AldicError):
        api.funIntegerSearch(np.zeros((10, 10)), np.zeros((10, 10)), 3, [1, 10], [1, 10], 4, 2, 1)


def test_integer_search_quadtree_distance_rules():
    import pytest
    import aldic_b200 as A

    roi = {"gridx": [1, 64], "gridy": [1, 64]}
    base = {"gridxyROIRange": roi, "winsize": 16, "winstepsize": 8, "InitFFTSearchMethod": 1}
    f = np.zeros((64, 64))
    # no distance for this image: the reference prompts; here it raises before any device work
    with pytest.raises(A.AldicError):
        A.IntegerSearchQuadtree(f, f, None, dict(base, TemporalSearchDistance=5), -1)
    with pytest.raises(A.AldicError):
        A.IntegerSearchQuadtree(f, f, None, dict(base, StereoSearchDistance=5), 2)
    with pytest.raises(A.AldicError):
        A.IntegerSearchQuadtree(f, f, None, dict(base, InitFFTSearchMethod=0, NewFFTSearchDistance=5), 2)


def _mesh_setup_loops(x, y):
    # the reference's loops (func/MeshSetUp.m), written out one entry at a time
    M, N = x.shape[1], x.shape[0]
    xt, yt = x.T, y.T
    cf = np.zeros((M * N, 2))
    for i in range(M * N):
        cf[i] = [xt.ravel(order="F")[i], yt.ravel(order="F")[i]]
    ef = np.zeros(((M - 1) * (N - 1), 4), dtype=np.int64)
    for j in range(1, N):
        for i in range(1, M):
            ef[(j - 1) * (M - 1) + i - 1] = [(j - 1) * M + i, (j - 1) * M + i + 1, j * M + i + 1, j * M + i]
    return cf, ef


def test_mesh_setup_matches_the_reference_loops():
    import aldic_b200 as A

    xl = np.arange(1, 120 - 20 - 8 + 1, 8) + 10.0
    yl = np.arange(1, 90 - 20 - 8 + 1, 8) + 10.0
    X, Y = np.meshgrid(xl, yl)           # nY x nX, as funIntegerSearch returns them
    D = A.MeshSetUp(X, Y, {"winstepsize": 8, "ImgSize": [120, 90]})
    cf, ef = _mesh_setup_loops(X, Y)
    assert np.array_equal(D["coordinatesFEM"], cf) and np.array_equal(D["elementsFEM"], ef)
    assert D["M"] == len(xl) and D["N"] == len(yl)
    assert np.array_equal(D["coordinatesFEMWorld"][:, 1], 91 - cf[:, 1])
    # the node list is the XList-fastest mesh the pipelines use
    assert D["coordinatesFEM"][1, 0] - D["coordinatesFEM"][0, 0] == 8


def test_integer_search_quadtree_zero_initial_guess():
    import aldic_b200 as A

    para = {"InitFFTSearchMethod": 3, "gridxyROIRange": {"gridx": [11, 60], "gridy": [5, 40]}, "winstepsize": 8}
    p2, x0, y0, u, v, cc = A.IntegerSearchQuadtree(None, None, None, para, 2)
    xs, ys = np.arange(11, 61, 8), np.arange(5, 41, 8)   # MATLAB gridx(1):step:gridx(2)
    assert x0.shape == (ys.size, xs.size) and np.array_equal(x0[0], xs) and np.array_equal(y0[:, 0], ys)
    assert not u.any() and not v.any() and (cc["max"] == 1).all()
    assert list(p2["SizeOfFFTSearchRegion"]) == [0, 0] and p2["InitFFTSearchMethod"] == 3
    with pytest.raises(A.AldicError):
        A.IntegerSearchQuadtree(None, None, None, dict(para, InitFFTSearchMethod=2), 2)


def test_organize_matched_pairs():
    import aldic_b200 as A

    C = np.array([[10.0, 20.0], [30.0, 40.0], [50.0, 60.0]])
    Cr = C + [[5.0, 1.0]]
    RD_L = {"ResultFEMeshEachFrame": [{"coordinatesFEM": C}],
            "ResultDisp": [{"U": np.array([[1.0, 2.0]] * 3)}, {"U": np.array([1.5, 2.5] * 3)}]}
    RD_R = {"Coordinates_corr": Cr, "ResultDisp": [{"U": np.array([[0.5, -1.0]] * 3)}, {"U": np.zeros(6)}]}
    P = A.organizeMatchedPairds_quadtree_ST1(RD_L, RD_R, {})
    assert len(P) == 3 and all(p.shape == (3, 4) for p in P)
    assert np.array_equal(P[0], np.concatenate([C, Cr], 1))
    assert np.array_equal(P[1][:, :2], C + [1.0, 2.0]) and np.array_equal(P[1][:, 2:], Cr + [0.5, -1.0])
    assert np.array_equal(P[2][:, :2], C + [1.5, 2.5]) and np.array_equal(P[2][:, 2:], Cr)


def test_learned_pipeline_order(monkeypatch):
    """LearnedPipeline (two contexts, one stream): each push loads and submits a frame on the
    other context before completing the previous frame (the host's wait for its fallback
    count), returns that previous frame, and flush completes the last one."""
    from aldic_b200 import learned as L

    log = []

    class FakeInit:
        def __init__(self, net, ctx, *args, stream=None, **kw):
            self.ctx, self.stream, self.n_fallback = ctx, stream, 0

        def submit(self):
            log.append(("submit", self.ctx))

        def complete(self):
            log.append(("complete", self.ctx))
            return 0

    monkeypatch.setattr(L, "LearnedInit", FakeInit)
    with pytest.raises(ValueError):
        L.LearnedPipeline("net", ["A"], 16, [1, 99], [1, 99], 32, 16, 1e-3)
    pipe = L.LearnedPipeline("net", ["A", "B"], 16, [1, 99], [1, 99], 32, 16, 1e-3)
    assert pipe.lis[1].stream is pipe.lis[0].stream
    done = [pipe.push(lambda ctx, k=k: log.append(("load", ctx, k))) for k in range(3)]
    last = pipe.flush()
    assert log == [("load", "A", 0), ("submit", "A"),
                   ("load", "B", 1), ("submit", "B"), ("complete", "A"),
                   ("load", "A", 2), ("submit", "A"), ("complete", "B"),
                   ("complete", "A")]
    assert done[0] is None and done[1].ctx == "A" and done[2].ctx == "B" and last.ctx == "A"
    assert pipe.flush() is None


def test_exact_integer_roi_statistics():
    """The arithmetic of roi_moment_int_kernel (prep.cu) on integer frames: exact sums
    S1 = sum x, S2 = sum x^2, the squared deviations (n S2 - S1^2) / n from the exact integer
    numerator split into 64-bit halves before the FP64 conversion, as the kernel does.  It
    equals numpy's two-pass FP64 mean and N-1 standard deviation to rounding, also where
    n S2 needs more than 64 bits (a u16 frame)."""
    import math

    rng = np.random.default_rng(0)
    for dtype, hi, shape in ((np.uint8, 256, (513, 257)), (np.uint16, 65536, (2048, 1024))):
        x = rng.integers(0, hi, size=shape).astype(dtype)
        n = x.size
        s1 = int(x.astype(np.int64).sum())
        s2 = int((x.astype(np.uint64) * x.astype(np.uint64)).sum(dtype=np.uint64))
        d = n * s2 - s1 * s1
        assert d >= 0
        if dtype == np.uint16:
            assert n * s2 >= 2 ** 64  # the high word is in use
        nd = float(d >> 64) * 18446744073709551616.0 + float(d & (2 ** 64 - 1))
        ssd = nd / n
        mean, sd = s1 / n, math.sqrt(ssd / (n - 1))
        xf = x.astype(np.float64)
        assert abs(mean - xf.mean()) <= 4e-16 * abs(xf.mean())
        assert abs(sd - xf.std(ddof=1)) <= 1e-14 * xf.std(ddof=1)
