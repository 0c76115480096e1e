"""The MATLAB MEX gateway (3d-stereo-aldic_b200/mex/aldic_mex.cpp), compiled against the test
stand-in for MATLAB's MEX runtime (tests/mex/), driven with mxArrays the way MATLAB calls it:
every command's outputs equal the direct C-ABI calls of the library on the same inputs
(GPU), masks may be logical or double, and argument errors come back as MATLAB errors
(CPU).  The MATLAB signatures follow func_quadtree/LocalICGNQuadtree.m:1-2,
func_quadtree/Subpb1Quadtree.m:1-2, func/funIntegerSearch.m:2, func/Init.m,
func/funRemoveOutliers.m, func_quadtree/Subpb2Quadtree.m,
func_quadtree/stereoReconstruction_quadtree.m:30-52 and ba_interp2_spline.cpp:418-435."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from aldic_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "mex", "libaldic_mex_host.so")
DOUBLE, INT32, UINT8, LOGICAL, CHAR = 6, 12, 9, 3, 4
_NP = {DOUBLE: np.float64, INT32: np.int32, UINT8: np.uint8, LOGICAL: np.uint8, CHAR: np.uint8}


class MxArg:
    """An mxArray built by Mex.arr (e.g. a logical mask), passed as it is."""

    def __init__(self, ptr):
        self.ptr = ptr


class Mex:
    """mexFunction of the gateway with numpy arguments and results (column-major)."""

    def __init__(self):
        if not os.path.exists(LIB):
            subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "mex")])
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.mexrt_array.restype = vp
        L.mexrt_array.argtypes = [C.c_int, C.c_int64, C.c_int64, vp]
        L.mexrt_string.restype = vp
        L.mexrt_string.argtypes = [C.c_char_p]
        L.mexrt_data.restype = vp
        L.mexrt_data.argtypes = [vp]
        for f in ("mexrt_rows", "mexrt_cols"):
            getattr(L, f).restype = C.c_int64
            getattr(L, f).argtypes = [vp]
        L.mexrt_class.restype = C.c_int
        L.mexrt_class.argtypes = [vp]
        L.mexrt_free.argtypes = [vp]
        L.mexrt_call.restype = C.c_int
        L.mexrt_call.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp), C.c_char_p, C.c_int]
        self.L = L

    def arr(self, a, cls=DOUBLE):
        """A new mxArray (an MxArg): strings as char arrays, everything else as an m x n array
        of class cls (scalars 1 x 1, vectors n x 1)."""
        return MxArg(self._new(a, cls))

    def _new(self, a, cls=DOUBLE):
        if isinstance(a, MxArg):
            return a.ptr
        if isinstance(a, str):
            return self.L.mexrt_string(a.encode())
        a = np.asarray(a, dtype=_NP[cls])
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(-1, 1)
        f = np.asfortranarray(a)
        return self.L.mexrt_array(cls, f.shape[0], f.shape[1], f.ctypes.data)

    def call(self, nout, *args):
        prhs = [self._new(a) for a in args]
        P = (C.c_void_p * len(prhs))(*prhs)
        O = (C.c_void_p * max(nout, 1))()
        err = C.create_string_buffer(1024)
        rc = self.L.mexrt_call(nout, O, len(prhs), P, err, len(err))
        for p in prhs:
            self.L.mexrt_free(p)
        if rc:
            raise RuntimeError(err.value.decode())
        outs = []
        for k in range(nout):
            p = O[k]
            m, n, cls = self.L.mexrt_rows(p), self.L.mexrt_cols(p), self.L.mexrt_class(p)
            dt = np.dtype(_NP[cls])
            buf = (C.c_char * (m * n * dt.itemsize)).from_address(self.L.mexrt_data(p))
            outs.append(np.frombuffer(buf, dtype=dt).reshape((m, n), order="F").copy())
            self.L.mexrt_free(p)
        return outs


def test_gateway_builds_and_rejects_bad_calls():
    # CPU: the gateway compiles against the MEX API, exports mexFunction, and argument errors
    # unwind as MATLAB errors before any device work
    mx = Mex()
    assert hasattr(mx.L, "mexFunction")
    with pytest.raises(RuntimeError, match="command string"):
        mx.call(1, np.zeros(3))


@pytest.fixture(scope="module")
def mx():
    m = Mex()
    yield m
    m.L.mexrt_exit()


@pytest.mark.gpu
def test_gateway_icgn_commands_match_the_c_abi(mx):
    import aldic_b200 as A

    ctx = A.Context(0)
    try:
        # LocalICGNQuadtree on a plate with a hole: logical and double masks
        sc = synth.plate_with_hole(size=384, hole_r=60.0, peak=2.0, sin_amp=0.3, sin_wl=120.0)
        M, N = sc.ref.shape
        ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
        ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
        ctx.set_mask(sc.mask)
        ctx.compute_gradients()
        f, g, gx, gy = (ctx.get_state(k) for k in range(4))
        xs = np.arange(20, 370, 8.0)
        X, Y = np.meshgrid(xs, xs, indexing="ij")
        coords = np.stack([X.ravel(), Y.ravel()], 1)
        tu, tv = sc.disp(coords[:, 0], coords[:, 1])
        U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
        ctx.load_image(0, f)
        ctx.load_image(1, g)
        ctx.set_gradients(gx, gy)
        want = ctx.local_icgn(1, coords, U0, 24, 1e-3)
        for mask_arg in (mx.arr(sc.mask != 0, LOGICAL), sc.mask.astype(np.float64)):
            U, F, H, conv, mark = mx.call(5, "local_icgn_quadtree", U0, coords, gx, gy, mask_arg, f, g, 24, 1e-3)
            assert np.array_equal(conv.ravel(), want["conv"])
            assert np.array_equal(U.ravel(), want["U"], equal_nan=True)
            assert np.array_equal(F.ravel(), want["F"], equal_nan=True)
            assert np.array_equal(H, want["H"])
            assert np.array_equal(mark.ravel(), want["markHole"])
        # Subpb1Quadtree with per-subset windows, right after (the frame stays loaded)
        n = len(coords)
        rng = np.random.default_rng(0)
        UOld = np.stack([tu, tv], 1).ravel() + rng.normal(0, 0.2, 2 * n)
        FOld = np.tile([0.005, 0.0, 0.0, -0.002], n)
        vdual = rng.normal(0, 0.05, 2 * n)
        wl = np.full((n, 2), 24, dtype=np.int32)
        want = ctx.subpb1(1, coords, UOld, FOld, vdual, 1e-3, 1e-3, winsize=24, winsize_list=wl)
        U, conv = mx.call(2, "subpb1_quadtree", UOld, FOld, vdual, coords, gx, gy, mx.arr(sc.mask != 0, LOGICAL), f,
                          g, 1e-3, wl.astype(np.float64), 1e-3)
        assert np.array_equal(conv.ravel(), want["conv"])
        assert np.array_equal(U.ravel(), want["U"], equal_nan=True)
        # LocalICGN and Subpb1 (uniform) on the affine scene
        sc = synth.temporal_affine()
        M, N = sc.ref.shape
        ctx.load_image_raw(0, sc.ref, [1, M], [1, N])
        ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
        ctx.set_mask(None)
        ctx.compute_gradients()
        f, g, gx, gy = (ctx.get_state(k) for k in range(4))
        ctx.load_image(0, f)
        ctx.load_image(1, g)
        ctx.set_gradients(gx, gy)
        r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
        x, y, u, v, phi = mx.call(5, "integer_search", f, g, [10, 10], [1, M], [1, N], 30, 16)
        for k, o in zip(("x", "y", "u", "v", "phi"), (x, y, u, v, phi)):
            assert np.array_equal(o, r[k], equal_nan=True), k
        coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
        U0 = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
        ctx.load_image(0, f)
        ctx.load_image(1, g)
        ctx.set_gradients(gx, gy)
        want = ctx.local_icgn(0, coords, U0, 30, 1e-3)
        U, F, H, conv = mx.call(4, "local_icgn", U0, coords, gx, gy, f, g, 30, 1e-3)
        assert np.array_equal(conv.ravel(), want["conv"])
        assert np.array_equal(U.ravel(), want["U"], equal_nan=True)
        assert np.array_equal(H, want["H"])
        n = len(coords)
        FOld = np.nan_to_num(want["F"])
        vdual = np.zeros(2 * n)
        want1 = ctx.subpb1(0, coords, np.nan_to_num(want["U"]), FOld, vdual, 1e-3, 1e-3, winsize=30,
                           HPar=want["H"])
        U, conv = mx.call(2, "subpb1", np.nan_to_num(want["U"]), FOld, vdual, coords, gx, gy, f, g, 1e-3, want["H"],
                          30, 1e-3)
        assert np.array_equal(conv.ravel(), want1["conv"])
        assert np.array_equal(U.ravel(), want1["U"], equal_nan=True)
        # Init and the bad-point removal on the search grids
        assert np.array_equal(mx.call(1, "init", r["u"], r["v"], 0)[0].ravel(), ctx.init_u0(r["u"], r["v"]))
        uo, vo = ctx.remove_outliers(r["u"].copy(), r["v"].copy(), 100.0)
        gu, gv = mx.call(2, "remove_outliers", r["u"], r["v"], 100.0)
        assert np.array_equal(gu, uo, equal_nan=True) and np.array_equal(gv, vo, equal_nan=True)
        # ba_interp2_spline(F, X, Y)
        rng = np.random.default_rng(5)
        Xq, Yq = rng.uniform(3, N - 3, (40, 25)), rng.uniform(3, M - 3, (40, 25))
        (Z,) = mx.call(1, "interp2", g, Xq, Yq)
        ctx.load_image(1, g)
        assert np.array_equal(Z, ctx.interp2(1, Xq, Yq))
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gateway_global_step_and_reconstruction_match_the_c_abi(mx):
    import aldic_b200 as A
    from test_subpb2_host import quadtree_mesh

    ctx = A.Context(0)
    try:
        Cc, E = quadtree_mesh(7, {(1, 1), (2, 1), (4, 4), (5, 2)})
        n = Cc.shape[0]
        rng = np.random.default_rng(11)
        U = 3.0 + rng.standard_normal(2 * n)
        F = 0.01 * rng.standard_normal(4 * n)
        dirichlet = [1, 5, 9]
        want = ctx.subpb2(Cc, E, 2, 0.05, 1e-3, U, F, dirichlet=dirichlet)
        (got,) = mx.call(1, "subpb2", Cc, np.asarray(E, np.float64), np.asarray(dirichlet, np.float64), 2, 0.05, 1e-3,
                         U, F, 0.0)
        assert np.array_equal(got.ravel(), want)
        K = np.array([[4000.0, 0.5, 1024.5], [0, 4010.0, 1000.2], [0, 0, 1]])
        pts = rng.uniform(1, 2048, (500, 2))
        (und,) = mx.call(1, "undistort", pts, K, [-0.12, 0.05, -0.01], [1e-3, -5e-4])
        assert np.array_equal(und, ctx.undistort_points(pts, K, [-0.12, 0.05, -0.01], [1e-3, -5e-4]))
        sc = synth.stereo_pair(seed=3, size=256, f=500.0)
        xy = rng.uniform(60, 200, (400, 2))
        pairs = np.hstack([xy, synth.stereo_truth(sc, xy)["right0"]])
        xyz, err = mx.call(2, "triangulate", pairs, sc.KL, sc.KR, sc.R_rl, np.ravel(sc.T_rl))
        wx, we = ctx.triangulate(pairs, sc.KL, sc.KR, sc.R_rl, sc.T_rl)
        assert np.array_equal(xyz, wx) and np.array_equal(err.ravel(), we)
        with pytest.raises(RuntimeError, match="unknown command"):
            mx.call(1, "no_such_command")
    finally:
        ctx.close()
