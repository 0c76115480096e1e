"""CPU check of the stereo match driver's glue (StereoMatch_STAQ).

The driver composes the library's calls (gradients, whole-field search, bad-point removal,
Init, IC-GN) with the host steps (MeshSetUp, GenerateQuadtreeMesh, the fills).  Here it runs
on a stand-in context whose device calls are the oracle's restatements, so the test checks
the order of the steps, the arguments passed between them and the outputs' layout, without
a GPU; the device calls themselves are checked against the oracle by the GPU tests.
"""
import numpy as np

import oracle as O
from aldic_b200 import synth


class OracleContext:
    """The Context methods the MATLAB-named drivers call, restated by the oracle."""

    def __init__(self):
        self.img = [None, None]
        self.mask = None
        self.g = (None, None)

    def load_image(self, slot, img):
        self.img[slot] = np.asarray(img, dtype=np.float64)

    def set_mask(self, mask):
        self.mask = None if mask is None else np.asarray(mask, dtype=np.float64)

    def compute_gradients(self):
        self.g = O.gradient(self.img[0], self.mask)

    def set_gradients(self, dfdx, dfdy):
        self.g = (np.asarray(dfdx, dtype=np.float64), np.asarray(dfdy, dtype=np.float64))

    def get_state(self, what):
        return [self.img[0], self.img[1], self.g[0], self.g[1]][what]

    def integer_search(self, search, gridx, gridy, winsize, step):
        return O.integer_search(self.img[0], self.img[1], list(np.ravel(search)), gridx, gridy, winsize, step)

    def remove_outliers(self, u, v, thr=100.0, maxit=0, info=False):
        u2, v2, _ = O.remove_outliers(u, v, thr)
        return u2, v2

    def init_u0(self, u, v, out=None, index=0):
        return O.init_u0(u, v, index)

    def subpb1(self, variant, coords, UOld, FOld, vdual, mu, tol, winsize=0, winsize_list=None, HPar=None, out=None):
        frame = O.Frame(self.img[0], self.img[1], self.mask, self.g[0], self.g[1])
        wl = None if winsize_list is None else np.asarray(winsize_list).reshape(-1, 2)
        return O.subpb1(frame, np.asarray(coords, dtype=np.float64), np.asarray(UOld, dtype=np.float64),
                        np.asarray(FOld, dtype=np.float64), np.asarray(vdual, dtype=np.float64), mu, tol,
                        winsize=winsize, winsize_list=wl, HPar=HPar, variant=variant)

    def subpb2(self, coords, elements, order, beta, mu, U, F, alpha=0.0, dirichlet=None, **kw):
        return O.subpb2_quadtree(coords, elements, order, beta, mu, U, F, alpha=alpha,
                                 dirichlet=() if dirichlet is None else dirichlet)

    def triangulate(self, pairs, KL, KR, R, T, out=None):
        return O.triangulate(pairs, KL, KR, R, T)

    def undistort_points(self, pts, K, radial, tangential=None):
        return O.undistort_points(pts, K, radial, tangential)

    def local_icgn(self, variant, coords, U0, winsize, tol, **kw):
        frame = O.Frame(self.img[0], self.img[1], self.mask, self.g[0], self.g[1])
        return O.local_icgn(frame, np.asarray(coords, dtype=np.float64), np.asarray(U0, dtype=np.float64), winsize,
                            tol, variant=variant)


def test_stereo_match_driver_on_the_oracle():
    import aldic_b200 as A

    O.build()
    sc = synth.temporal_affine(seed=3, M=192, N=176, n_speckles=1200, u=2.6, v=-1.4)
    M, N = sc.ref.shape
    mask = np.ones((M, N))
    X, Y = np.meshgrid(np.arange(1, M + 1), np.arange(1, N + 1), indexing="ij")
    mask[(X - 96) ** 2 + (Y - 90) ** 2 < 24 ** 2] = 0
    para = {"winsize": 20, "winstepsize": 16, "winsizeMin": 4, "StereoSearchDistance": 6, "ImgSize": [M, N],
            "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "ImgRefMask": mask}
    info, RD_L, RD_R = A.StereoMatch_STAQ({}, {}, sc.ref.astype(float), sc.deff.astype(float), None, mask, mask,
                                          para, {}, 1, ctx=OracleContext())
    C = info["ResultFEMeshEachFrame"]["coordinatesFEM"]
    E = info["ResultFEMeshEachFrame"]["elementsFEM"]
    assert E.shape[1] == 8 and (E[:, 4:] > 0).any()               # a quadtree with hanging nodes
    assert info["U"].shape == (2 * C.shape[0],) and np.isfinite(info["U"]).all()   # filled
    assert np.array_equal(RD_R["Coordinates_corr"], C + info["U"].reshape(-1, 2))
    # away from the hole and the border, the match is the true displacement
    tu, tv = sc.disp(C[:, 0], C[:, 1])
    ix = np.floor(C[:, 0] + 0.5).astype(int) - 1
    iy = np.floor(C[:, 1] + 0.5).astype(int) - 1
    far = (np.hypot(C[:, 0] - 96, C[:, 1] - 90) > 40) & (C[:, 0] > 20) & (C[:, 0] < M - 20) & \
          (C[:, 1] > 20) & (C[:, 1] < N - 20) & (mask[ix, iy] > 0)
    err = np.hypot(info["U"][0::2] - tu, info["U"][1::2] - tv)[far]
    assert far.sum() > 20 and np.median(err) < 0.02
    # CalPointsNum is the search grid's shape, the uniform mesh's node count
    assert int(np.prod(info["CalPointsNum"])) == info["ResultFEMesh"]["coordinatesFEM"].shape[0]


def test_aldic_frame_on_the_oracle():
    """One ALDIC frame (TemporalMatch_quadtree_ST1 sections 3-6) on a masked plate, the
    device calls restated by the oracle: every step runs, the global step's beta comes from
    the tuning rule, and the final displacements match the plate's known field."""
    import aldic_b200 as A

    O.build()
    sc = synth.plate_with_hole(size=256, hole_r=40.0, peak=1.5, sin_amp=0.2, sin_wl=100.0)
    M, N = sc.ref.shape
    para = {"winsize": 24, "winstepsize": 16, "winsizeMin": 8, "TemporalSearchDistance": 6, "ImgSize": [M, N],
            "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "ImgRefMask": sc.mask}
    ctx = OracleContext()
    r = A.ALDICFrameQuadtree(sc.ref.astype(float) * sc.mask, sc.deff.astype(float), sc.mask, para, 2, ctx=ctx)
    mesh = r["DICmesh"]
    C = mesh["coordinatesFEM"]
    assert r["U"].shape == (2 * C.shape[0],) and mesh["elementsFEM"].shape[1] == 8
    step = 16.0
    betas = [c * step ** 2 * 1e-3 for c in (1e-3, 1e-2, 1e-1)]
    assert betas[0] <= r["beta"] <= betas[2]
    used = np.unique(mesh["elementsFEM"][mesh["elementsFEM"] > 0]) - 1
    tu, tv = sc.disp(C[:, 0], C[:, 1])
    ix = np.floor(C[:, 0] + 0.5).astype(int) - 1
    iy = np.floor(C[:, 1] + 0.5).astype(int) - 1
    inside = np.zeros(C.shape[0], bool)
    inside[used] = True
    inside &= (sc.mask[ix, iy] > 0) & (C[:, 0] > 24) & (C[:, 0] < M - 24) & (C[:, 1] > 24) & (C[:, 1] < N - 24)
    err = np.hypot(r["U"][0::2] - tu, r["U"][1::2] - tv)[inside]
    assert inside.sum() > 30 and np.isfinite(err).all() and np.median(err) < 0.05



def test_temporal_match_driver_on_the_oracle():
    """TemporalMatch_quadtree_ST1 (accumulative) over three frames with one reference
    speckle pattern, both camera forms and the 'reuseLast' seed: the device calls restated
    by the oracle, the fields recovered at the first frame's mesh (camera0) and at given
    matched points (notCamera0)."""
    import aldic_b200 as A

    O.build()
    M = N = 176
    frames = [synth.temporal_affine(seed=5, M=M, N=N, n_speckles=1100, u=u, v=v, dudx=0.001, dvdy=-0.001)
              for u, v in ((1.6, -0.8), (2.9, -1.7))]
    imgs = [frames[0].ref.astype(float)] + [f.deff.astype(float) for f in frames]
    mask = np.ones((M, N))
    X, Y = np.meshgrid(np.arange(1, M + 1), np.arange(1, N + 1), indexing="ij")
    mask[(X - 90) ** 2 + (Y - 84) ** 2 < 22 ** 2] = 0
    para = {"winsize": 20, "winstepsize": 16, "winsizeMin": 8, "TemporalSearchDistance": 6, "ImgSize": [M, N],
            "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "TemporalInitGuess": "reuseLast"}
    ctx = OracleContext()
    RD = A.TemporalMatch_quadtree_ST1(para, None, [mask] * 3, imgs, {}, None, "camera0", 1, ctx=ctx)
    C = RD["ResultFEMeshEachFrame"][0]["coordinatesFEM"]
    assert len(RD["ResultDisp"]) == 2 and RD["ResultDisp"][1]["U"].shape == (C.shape[0], 2)
    ix = np.floor(C[:, 0] + 0.5).astype(int) - 1
    iy = np.floor(C[:, 1] + 0.5).astype(int) - 1
    good = (mask[ix, iy] > 0) & (np.hypot(C[:, 0] - 90, C[:, 1] - 84) > 36) & (C[:, 0] > 20) & (C[:, 0] < M - 20) \
        & (C[:, 1] > 20) & (C[:, 1] < N - 20)
    for k, f in enumerate(frames):
        tu, tv = f.disp(C[:, 0], C[:, 1])
        U = RD["ResultDisp"][k]["U"]
        assert np.median(np.hypot(U[good, 0] - tu[good], U[good, 1] - tv[good])) < 0.03, k
    # the second camera's form: the field carried to matched points inside the mesh
    inner = good & (C[:, 0] < C[:, 0].max() - 1) & (C[:, 1] < C[:, 1].max() - 1)
    pts = C[inner][:20] + [0.5, 0.25]  # inside the mesh's hull
    RDr = A.TemporalMatch_quadtree_ST1(para, None, [mask] * 3, imgs, {"Coordinates_corr": pts}, None, "notCamera0", 1,
                                       ctx=ctx)
    Ur = RDr["ResultDisp"][1]["U"]
    tu, tv = frames[1].disp(pts[:, 0], pts[:, 1])
    assert Ur.shape == (20, 2) and np.median(np.hypot(Ur[:, 0] - tu, Ur[:, 1] - tv)) < 0.03
    assert len(RDr["ResultDisp_corr"]) == 2


def test_stereo_pipeline_end_to_end_on_the_oracle():
    """The reference's stereo sequence, driver by driver: StereoMatch_STAQ on the first pair,
    TemporalMatch_quadtree_ST1 for the left camera and for the right one (its field at the
    stereo-matched points), organizeMatchedPairds_quadtree_ST1 and
    stereoReconstruction_quadtree; the plane's rigid 3-D motion comes back."""
    import aldic_b200 as A

    O.build()
    sc = synth.stereo_pair(seed=2, size=224, f=500.0, plane_half=320.0, motion_t=(1.0, -0.6, 3.0),
                           motion_rot=2e-3)
    L = [im.astype(float) for im in sc.L]
    R = [im.astype(float) for im in sc.R]
    M, N = L[0].shape
    ones = np.ones((M, N))
    para = {"winsize": 20, "winstepsize": 16, "winsizeMin": 8, "StereoSearchDistance": 14,
            "TemporalSearchDistance": 6, "ImgSize": [M, N], "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]},
            "ImgRefMask": ones}
    ctx = OracleContext()
    info, RD_L, RD_R = A.StereoMatch_STAQ({}, {}, L[0], R[0], None, ones, ones, para, {}, 1, ctx=ctx)
    RD_L = A.TemporalMatch_quadtree_ST1(para, None, [ones, ones], L, RD_L, info, "camera0", 1, ctx=ctx)
    RD_R = A.TemporalMatch_quadtree_ST1(para, None, [ones, ones], R, RD_R, info, "notCamera0", 1, ctx=ctx)
    assert np.array_equal(RD_L["ResultFEMeshEachFrame"][0]["coordinatesFEM"],
                          info["ResultFEMeshEachFrame"]["coordinatesFEM"])  # one mesh for both drivers
    pairs = A.organizeMatchedPairds_quadtree_ST1(RD_L, RD_R, para)
    cam = {"KL": sc.KL, "KR": sc.KR, "R": sc.R_rl, "T": sc.T_rl}
    final, errs = A.stereoReconstruction_quadtree(pairs, cam, ctx=ctx)
    C = RD_L["ResultFEMeshEachFrame"][0]["coordinatesFEM"]
    t = synth.stereo_truth(sc, C, 1)
    inner = (C[:, 0] > 30) & (C[:, 0] < M - 30) & (C[:, 1] > 30) & (C[:, 1] < N - 30)

    def med(e):
        return float(np.nanmedian(np.linalg.norm(e, axis=1)[inner]))

    # each stage in pixels: the stereo match, the left and the right temporal fields
    Cr = RD_R["Coordinates_corr"]
    assert med(Cr - t["right0"]) < 0.06
    assert med(C + RD_L["ResultDisp"][0]["U"] - t["left1"]) < 0.06
    assert med(Cr + RD_R["ResultDisp"][0]["U"] - t["right1"]) < 0.06
    # in 3-D, left camera frame (P_L = K [I | 0]): ~6.7 mm of depth per pixel of disparity here
    X0 = synth.to_left_camera_frame(sc, t["xyz0"])
    X1 = synth.to_left_camera_frame(sc, t["xyz1"])
    ok = inner & np.isfinite(final["Displacement"][1]).all(1)
    assert ok.sum() > 20
    assert np.median(np.linalg.norm(final["Coordinates"][0][ok] - X0[ok], axis=1)) < 1.0      # mm at ~1 m
    d = np.linalg.norm(final["Displacement"][1][ok] - (X1 - X0)[ok], axis=1)
    assert np.median(d) < 0.25                                                                 # mm of ~3.2 mm


def test_local_icgn_uniform_driver_fills_u_and_f():
    """LocalICGN (uniform mesh) as the reference returns it: bad points (here subsets whose
    window leaves the image) filled in U and in F from the good ones."""
    import aldic_b200 as A

    O.build()
    sc = synth.temporal_affine(seed=7, M=160, N=160, n_speckles=900, u=2.2, v=-1.1)
    M, N = sc.ref.shape
    ctx = OracleContext()
    Df = A.funImgGradient(sc.ref.astype(float), ctx=ctx)
    xs = np.arange(8.0, 156.0, 12.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    C = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(C[:, 0], C[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    U, F, H, t, conv, nbad = A.LocalICGN(U0, C, Df, sc.ref.astype(float), sc.deff.astype(float), {"winsize": 20},
                                         ctx=ctx)
    Un, Fn, *_ = A.LocalICGN(U0, C, Df, sc.ref.astype(float), sc.deff.astype(float), {"winsize": 20}, ctx=ctx,
                             fill=False)
    bad = np.isnan(Un[0::2])
    # failed subsets (code -1 at the border) and, by the uniform rule, iteration-count outliers
    assert bad.sum() >= nbad >= 5
    assert np.isfinite(U).all() and np.isfinite(F).all()
    assert np.array_equal(U.reshape(-1, 2)[~bad], Un.reshape(-1, 2)[~bad])
    # the filled border values continue the affine field
    err = np.hypot(U[0::2] - tu, U[1::2] - tv)[bad]
    assert np.median(err) < 0.05


def test_temporal_match_incremental_mode_accumulates():
    """The incremental mode: each frame against the previous one, the increments carried to
    the tracked points and summed; frame 3's accumulated field is the total displacement."""
    import aldic_b200 as A

    O.build()
    M = N = 176
    frames = [synth.temporal_affine(seed=5, M=M, N=N, n_speckles=1100, u=u, v=v, dudx=0.001, dvdy=-0.001)
              for u, v in ((1.6, -0.8), (2.9, -1.7))]
    imgs = [frames[0].ref.astype(float)] + [f.deff.astype(float) for f in frames]
    ones = np.ones((M, N))
    para = {"winsize": 20, "winstepsize": 16, "winsizeMin": 8, "TemporalSearchDistance": 6, "ImgSize": [M, N],
            "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "DICIncOrNot": 1}
    RD = A.TemporalMatch_quadtree_ST1(para, None, [ones] * 3, imgs, {}, None, "camera0", 1, ctx=OracleContext())
    assert len(RD["ResultDisp_inc"]) == 2 and len(RD["ResultFEMeshEachFrame"]) == 2
    C = RD["ResultFEMeshEachFrame"][0]["coordinatesFEM"]
    inner = (C[:, 0] > 24) & (C[:, 0] < M - 40) & (C[:, 1] > 24) & (C[:, 1] < N - 40)
    for k, f in enumerate(frames):
        tu, tv = f.disp(C[:, 0], C[:, 1])
        U = RD["ResultDisp"][k]["U"]
        e = np.hypot(U[:, 0] - tu, U[:, 1] - tv)[inner]
        assert np.isfinite(e).sum() > 20 and np.nanmedian(e) < 0.05, k


def test_uniform_subpb1_driver_ends_with_the_gridfit_surface():
    """Subpb1 (uniform) as the reference returns it: every node on the gridfit 'springs'
    surface of the good nodes (func/Subpb1.m:186-199)."""
    import aldic_b200 as A
    from aldic_b200.fill import gridfit_springs

    O.build()
    sc = synth.temporal_affine(seed=8, M=160, N=160, n_speckles=900, u=1.7, v=-0.9)
    ctx = OracleContext()
    Df = A.funImgGradient(sc.ref.astype(float), ctx=ctx)
    xs = np.arange(20.0, 141.0, 12.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    C = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(C[:, 0], C[:, 1])
    U0 = np.stack([tu, tv], 1).ravel()
    F0 = np.tile([sc.dudx, 0.0, 0.0, sc.dvdy], len(C))
    args = (U0, F0, np.zeros(4 * len(C)), np.zeros(2 * len(C)), C, Df, sc.ref.astype(float), sc.deff.astype(float),
            1e-3, 0.0, None, 1, {"winsize": 20})
    U, *_ = A.Subpb1(*args, ctx=ctx)
    Un, *_ = A.Subpb1(*args, ctx=ctx, fill=False)
    assert np.isfinite(U).all()
    zg = gridfit_springs(C[:, 0], C[:, 1], Un[0::2], xs, xs)
    assert np.abs(U[0::2] - zg[np.searchsorted(xs, C[:, 1]), np.searchsorted(xs, C[:, 0])]).max() < 1e-12
    assert np.median(np.hypot(U[0::2] - tu, U[1::2] - tv)) < 0.02


def test_aldic_frame_with_displacement_smoothing():
    """The ALDIC frame with the optional smoothing switched on (Smooth2DTimes 1,
    DispSmoothness 5e-4): every step runs and the field still matches the plate's."""
    import aldic_b200 as A

    O.build()
    sc = synth.plate_with_hole(size=256, hole_r=40.0, peak=1.5, sin_amp=0.2, sin_wl=100.0)
    M, N = sc.ref.shape
    para = {"winsize": 24, "winstepsize": 16, "winsizeMin": 8, "TemporalSearchDistance": 6, "ImgSize": [M, N],
            "gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "ImgRefMask": sc.mask, "Smooth2DTimes": 1,
            "DispSmoothness": 5e-4, "DispFilterStd": 0, "DispFilterSize": 0}
    r = A.ALDICFrameQuadtree(sc.ref.astype(float) * sc.mask, sc.deff.astype(float), sc.mask, para, 2,
                             ctx=OracleContext())
    C = r["DICmesh"]["coordinatesFEM"]
    tu, tv = sc.disp(C[:, 0], C[:, 1])
    ix = np.floor(C[:, 0] + 0.5).astype(int) - 1
    iy = np.floor(C[:, 1] + 0.5).astype(int) - 1
    inside = (sc.mask[ix, iy] > 0) & (C[:, 0] > 24) & (C[:, 0] < M - 24) & (C[:, 1] > 24) & (C[:, 1] < N - 24)
    err = np.hypot(r["U"][0::2] - tu, r["U"][1::2] - tv)[inside]
    assert np.isfinite(err).all() and np.median(err) < 0.08


def test_reconstruction_undistorts_first():
    """stereoReconstruction_quadtree with lens distortion: pairs pushed through each camera's
    lens model and reconstructed with its coefficients give the same 3-D points as the
    undistorted pairs without them (funUndistortPoints, then triangulate)."""
    import aldic_b200 as A

    sc = synth.stereo_pair(seed=2, size=224, f=500.0, plane_half=320.0)
    xs = np.arange(40.0, 190.0, 25.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    C = np.stack([X.ravel(), Y.ravel()], 1)
    t = synth.stereo_truth(sc, C)
    pairs = [np.concatenate([C, t["right0"]], 1)]
    cam = {"KL": sc.KL, "KR": sc.KR, "R": sc.R_rl, "T": sc.T_rl}
    ref, _ = A.stereoReconstruction_quadtree(pairs, cam, ctx=OracleContext())
    lens = dict(cam, radialL=[-0.08, 0.01], tangentialL=[1e-3, -5e-4], radialR=[0.05, -0.02, 0.003],
                tangentialR=[-8e-4, 2e-4])
    dpairs = [np.concatenate([O.distort_points(C, sc.KL, lens["radialL"], lens["tangentialL"]),
                              O.distort_points(t["right0"], sc.KR, lens["radialR"], lens["tangentialR"])], 1)]
    got, _ = A.stereoReconstruction_quadtree(dpairs, lens, ctx=OracleContext())
    assert np.abs(got["Coordinates"][0] - ref["Coordinates"][0]).max() < 1e-6
    assert np.abs(dpairs[0] - pairs[0]).max() > 0.1   # the lens model moved the points

