"""GPU parity tests: the CUDA path (through the C ABI) against the FP64 oracle on the
same seeded inputs.

Tolerances (FP32 interpolation/accumulation on the device, FP64 oracle):
  * normalised images, gradients, interpolation: 2e-6 relative to the data range;
  * integer search: u, v identical wherever the argmax is unambiguous; phi within 1e-6;
  * IC-GN / Subpb1: convergence flag identical on >= 99.9 % of subsets, u/v within
    1e-3 px on subsets both sides converged (the ALDIC bar), F within 1e-4;
  * triangulation: 1e-5 relative.
"""
import numpy as np
import pytest

import oracle as O
from aldic_b200 import synth

pytestmark = pytest.mark.gpu

UV_TOL = 1e-3
FLAG_RATE = 0.999


@pytest.fixture(scope="module")
def A():
    import aldic_b200

    return aldic_b200


@pytest.fixture(scope="module")
def ctx(A):
    c = A.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def affine():
    sc = synth.temporal_affine()
    return sc


def _load_raw(ctx, sc, mask=None):
    M, N = sc.ref.shape
    gx, gy = [1, M], [1, N]
    ctx.load_image_raw(0, sc.ref, gx, gy)
    ctx.load_image_raw(1, sc.deff, gx, gy)
    ctx.set_mask(mask)
    ctx.compute_gradients()


def _flag(conv):
    conv = np.asarray(conv)
    return (conv > 0) & (conv < 100)


def test_prep_parity(ctx, affine):
    sc = affine
    M, N = sc.ref.shape
    f, ms = O.normalize(sc.ref.astype(float), [1, M], [1, N])
    ms_g = ctx.load_image_raw(0, sc.ref, [1, M], [1, N])
    assert np.allclose(ms_g, ms, rtol=1e-13)
    assert np.max(np.abs(ctx.get_state(0) - f)) < 2e-6 * np.abs(f).max()
    mask = np.ones((M, N))
    mask[200:260, 300:350] = 0
    ctx.set_mask(mask)
    ctx.compute_gradients()
    gx, gy = O.gradient(ctx.get_state(0), mask)
    assert np.max(np.abs(ctx.get_state(2) - gx)) < 2e-6 * np.abs(gx).max()
    assert np.max(np.abs(ctx.get_state(3) - gy)) < 2e-6 * np.abs(gy).max()


def test_interp_matches_reference_golden(A, ctx):
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "interp_golden.npz"))
    for name in ("speckle", "ramp", "normalised"):
        F, X, Y, Z = g[f"{name}_F"], g[f"{name}_X"], g[f"{name}_Y"], g[f"{name}_Z"]
        z = A.ba_interp2_spline(F, X, Y, ctx=ctx)
        assert np.max(np.abs(z - Z)) <= 2e-6 * np.abs(F).max(), name


def test_integer_search_parity_affine(ctx, affine):
    sc = affine
    _load_raw(ctx, sc)
    M, N = sc.ref.shape
    f, g = ctx.get_state(0), ctx.get_state(1)
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    ro = O.integer_search(f, g, [10, 10], [1, M], [1, N], 30, 16)
    for k in ("x", "y", "u", "v"):
        assert np.array_equal(r[k], ro[k]), k
    assert np.nanmax(np.abs(r["phi"] - ro["phi"])) < 1e-6


def test_integer_search_edge_cases(ctx):
    # rectangular quirk [s0 s1 s0 s1], border clamps and a constant template -> NaN
    sc = synth.temporal_affine(M=200, N=180, n_speckles=500, u=4.2, v=2.6)
    ref = sc.ref.copy()
    ref[:40, :40] = 77  # flat patch: constant template at the origin
    sc2 = synth.AffineScene(ref=ref, deff=sc.deff, u0=sc.u0, v0=sc.v0, dudx=sc.dudx, dvdy=sc.dvdy, xc=sc.xc,
                            yc=sc.yc)
    _load_raw(ctx, sc2)
    f, g = ctx.get_state(0), ctx.get_state(1)
    for search, gx, gy, w, st in (([3, 7], [1, 200], [1, 180], 20, 12), ([6, 6], [5, 190], [9, 170], 16, 9),
                                  ([0, 0], [1, 200], [1, 180], 10, 20)):
        r = ctx.integer_search(search, gx, gy, w, st)
        ro = O.integer_search(f, g, search, gx, gy, w, st)
        assert np.array_equal(np.isnan(r["u"]), np.isnan(ro["u"]))
        ok = np.isfinite(ro["u"])
        assert np.array_equal(r["u"][ok], ro["u"][ok]) and np.array_equal(r["v"][ok], ro["v"][ok])
    assert np.isnan(ctx.integer_search([3, 7], [1, 200], [1, 180], 20, 12)["u"][0, 0])


@pytest.mark.parametrize("w,st,search,grid", [
    (40, 10, (12, 12), ([1, 330], [1, 300])),   # shared-product tile kernel, the stereo workload's shape
    (40, 10, (3, 9), ([7, 322], [4, 290])),     # same, rectangular search and border clamps
    (32, 16, (8, 8), ([1, 330], [1, 300])),     # tile kernel with REM = 1, Q = 2
    (24, 7, (5, 6), ([1, 330], [1, 300])),      # no tile kernel for this pair: per-subset kernel
])
def test_integer_search_parity_paths(ctx, w, st, search, grid):
    sc = synth.temporal_affine(M=330, N=300, n_speckles=1500, u=3.4, v=-2.7)
    _load_raw(ctx, sc)
    f, g = ctx.get_state(0), ctx.get_state(1)
    r = ctx.integer_search(list(search), grid[0], grid[1], w, st)
    ro = O.integer_search(f, g, list(search), grid[0], grid[1], w, st)
    assert np.array_equal(r["x"], ro["x"]) and np.array_equal(r["y"], ro["y"])
    assert np.array_equal(np.isnan(r["u"]), np.isnan(ro["u"]))
    ok = np.isfinite(ro["u"])
    assert ok.sum() > 50
    assert np.array_equal(r["u"][ok], ro["u"][ok]) and np.array_equal(r["v"][ok], ro["v"][ok])
    assert np.max(np.abs(r["phi"][ok] - ro["phi"][ok])) < 1e-6


def test_search_profiling_hook(ctx, affine):
    _load_raw(ctx, affine)
    M, N = affine.ref.shape
    ctx.set_profiling(True)
    ctx.profile_read()
    ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    ms, n = ctx.profile_read()
    ctx.set_profiling(False)
    assert n == 2 and ms > 0
    ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    assert ctx.profile_read() == (0.0, 0)


@pytest.mark.parametrize("variant", [0, 1])
def test_local_icgn_parity_affine(ctx, affine, variant):
    sc = affine
    _load_raw(ctx, sc, mask=np.ones(sc.ref.shape) if variant == 1 else None)
    M, N = sc.ref.shape
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0 = np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1).ravel()
    res = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
    ref = O.local_icgn(O.Frame(f, g, None if variant == 0 else np.ones_like(f), gx, gy), coords, U0, 30, 1e-3,
                       variant=variant)
    assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
    assert np.array_equal(res["conv"] == -1, ref["conv"] == -1)
    both = _flag(res["conv"]) & _flag(ref["conv"])
    assert both.sum() > 800
    du = np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both]
    assert du.max() < UV_TOL
    dF = np.abs(res["F"] - ref["F"]).reshape(-1, 4)[both]
    assert dF.max() < 1e-4
    Hr = ref["H"][both]
    assert np.max(np.abs(res["H"][both] - Hr) / (np.abs(Hr).max(axis=1, keepdims=True))) < 1e-5
    assert np.all(np.isnan(res["U"].reshape(-1, 2)[res["conv"] == -1]))


@pytest.mark.parametrize("variant", [0, 1])
def test_local_icgn_fp64_resolve_band(A, ctx, affine, variant):
    # band 0: every convergence test decided in FP32 (Kahan-compensated sums), the old bar;
    # a huge band: every subset re-solved from its initial guess by the FP64 kernel with the
    # reference's interpolation arithmetic on the same FP32 images as the oracle sees, so
    # codes are identical and U, F, H agree to FP64 rounding; the default band: codes equal
    sc = affine
    _load_raw(ctx, sc, mask=np.ones(sc.ref.shape) if variant == 1 else None)
    M, N = sc.ref.shape
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0 = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
    ref = O.local_icgn(O.Frame(f, g, None if variant == 0 else np.ones_like(f), gx, gy), coords, U0, 30, 1e-3,
                       variant=variant)
    ok = _flag(ref["conv"])
    try:
        ctx.set_fp64_band(0.0)
        r32 = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
        ctx.set_fp64_band(1e300)
        r64 = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
    finally:
        ctx.set_fp64_band(A.DEFAULT_FP64_BAND, A.DEFAULT_FP64_NOISE)
    rd = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
    both = _flag(r32["conv"]) & ok
    assert np.mean(_flag(r32["conv"]) == ok) >= FLAG_RATE
    assert np.abs(r32["U"] - ref["U"]).reshape(-1, 2)[both].max() < UV_TOL
    assert np.array_equal(r64["conv"], ref["conv"])
    assert np.array_equal(np.isnan(r64["U"]), np.isnan(ref["U"]))
    assert np.abs(r64["U"] - ref["U"]).reshape(-1, 2)[ok].max() < 1e-8
    assert np.abs(r64["F"] - ref["F"]).reshape(-1, 4)[ok].max() < 1e-9
    Hr = ref["H"][ok]
    assert np.max(np.abs(r64["H"][ok] - Hr) / np.abs(Hr).max(axis=1, keepdims=True)) < 1e-11
    assert np.array_equal(rd["conv"], ref["conv"])
    assert np.abs(rd["U"] - ref["U"]).reshape(-1, 2)[ok].max() < 1e-5
    with pytest.raises(Exception):
        ctx.set_fp64_band(-1.0)


def test_local_icgn_fp64_resolve_masked(A, ctx, hole):
    # the FP64 re-solve of masked subsets: bwselect regions, enlarged windows, the regrowth
    # rule and codes -1 / 102 / 103 all decided in FP64
    sc = hole
    M, N = sc.ref.shape
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(20, 370, 8.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    ref = O.local_icgn(O.Frame(f, g, sc.mask, gx, gy), coords, U0, 24, 1e-3, variant=1)
    try:
        ctx.set_fp64_band(1e300)
        r64 = ctx.local_icgn(1, coords, U0, 24, 1e-3)
    finally:
        ctx.set_fp64_band(A.DEFAULT_FP64_BAND, A.DEFAULT_FP64_NOISE)
    assert np.array_equal(r64["conv"], ref["conv"])
    assert np.array_equal(r64["markHole"], ref["markHole"])
    ok = _flag(ref["conv"])
    assert np.abs(r64["U"] - ref["U"]).reshape(-1, 2)[ok].max() < 1e-8


@pytest.mark.parametrize("variant", [0, 1])
def test_local_icgn_tma_staging_matches_gathers(A, ctx, affine, variant):
    # the warp passes' TMA-staged deformed windows give bit-identical results to the gather
    # path (same stencil operations, shared memory instead of the image); an iteration cap of
    # 2 also drives the multi-warp pass through its staged form
    sc = affine
    _load_raw(ctx, sc, mask=np.ones(sc.ref.shape) if variant == 1 else None)
    M, N = sc.ref.shape
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0 = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
    staging0 = ctx.get_option(A.OPT_STAGING)
    try:
        out = {}
        for cap in (8, 2):
            ctx.set_option(A.OPT_ITERATION_CAP, cap)
            for staging in (1, 0):
                ctx.set_option(A.OPT_STAGING, staging)
                out[cap, staging] = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
    finally:
        ctx.set_option(A.OPT_STAGING, staging0)
        ctx.set_option(A.OPT_ITERATION_CAP, A.DEFAULT_ITERATION_CAP)
    for cap in (8, 2):
        a, b = out[cap, 1], out[cap, 0]
        assert np.array_equal(a["conv"], b["conv"]), cap
        assert np.array_equal(a["U"], b["U"], equal_nan=True), cap
        assert np.array_equal(a["F"], b["F"], equal_nan=True), cap
    with pytest.raises(Exception):
        ctx.set_option(A.OPT_STAGING, 2)


def test_local_icgn_tma_staging_large_deformation(A, ctx):
    # a 6 % stretch and a 4 % contraction: boxes reload as the warp grows, and iterations whose
    # footprint outgrows the box gather from the image; still bit-identical to the gather path
    # and within the parity bar of the oracle
    sc = synth.temporal_affine(M=384, N=384, n_speckles=2400, u=2.3, v=-1.4, dudx=0.06, dvdy=-0.04)
    _load_raw(ctx, sc)
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(40, 345, 9.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    try:
        ctx.set_option(A.OPT_STAGING, 0)
        b = ctx.local_icgn(0, coords, U0, 40, 1e-3)
        ctx.set_option(A.OPT_STAGING, 1)
        a = ctx.local_icgn(0, coords, U0, 40, 1e-3)
    finally:
        ctx.set_option(A.OPT_STAGING, 0)
    assert np.array_equal(a["conv"], b["conv"])
    assert np.array_equal(a["U"], b["U"], equal_nan=True)
    ref = O.local_icgn(O.Frame(f, g, None, gx, gy), coords, U0, 40, 1e-3, variant=0)
    ok = _flag(ref["conv"])
    assert ok.sum() > 0.9 * len(ok)
    assert np.array_equal(a["conv"], ref["conv"])
    assert np.abs(a["U"] - ref["U"]).reshape(-1, 2)[ok].max() < UV_TOL


def test_autotuner_candidates_agree(A, affine):
    # the autotuner runs every candidate (IC-GN: staging x slow-pass warps x FP64 re-solve
    # threads x iteration cap;
    # search: tile kernel with 24 / 16 shift columns, direct kernel) on the call's inputs and
    # keeps the fastest of those whose results agree with the first; every candidate must
    # agree, and the tuned call's results equal an untuned call's
    c = A.Context(0)
    try:
        sc = affine
        _load_raw(c, sc)
        M, N = sc.ref.shape
        r0 = c.integer_search([10, 10], [1, M], [1, N], 30, 16)
        coords = np.stack([r0["x"].T.ravel(order="F"), r0["y"].T.ravel(order="F")], 1)
        U0 = np.nan_to_num(np.stack([r0["u"].T.ravel(order="F"), r0["v"].T.ravel(order="F")], 1)).ravel()
        w0 = c.local_icgn(0, coords, U0, 30, 1e-3)
        c.set_option(A.OPT_AUTOTUNE, 1)
        r1 = c.integer_search([10, 10], [1, M], [1, N], 30, 16)
        w1 = c.local_icgn(0, coords, U0, 30, 1e-3)
        w2 = c.local_icgn(0, coords, U0, 30, 1e-3)  # the cached choice, no timing
        rep = c.tuning_report()
        ks = [k for k in rep if k.startswith("search")]
        ki = [k for k in rep if k.startswith("icgn")]
        assert len(ks) == 1 and len(ki) == 1
        assert set(rep[ks[0]]["ms"]) == {"tile24", "tile16", "direct"}
        assert all(t > 0 for t in rep[ks[0]]["ms"].values())
        assert len(rep[ki[0]]["ms"]) == 16 and all(t > 0 for t in rep[ki[0]]["ms"].values())
        for k in ("u", "v"):
            assert np.array_equal(r0[k], r1[k], equal_nan=True)
        ok = _flag(w0["conv"])
        for w in (w1, w2):
            assert np.array_equal(w["conv"], w0["conv"])
            assert np.abs(w["U"] - w0["U"]).reshape(-1, 2)[ok].max() <= 1e-5
        # each search candidate set explicitly gives the same integer peaks
        c.set_option(A.OPT_AUTOTUNE, 0)
        for impl, chunk in ((1, 16), (1, 24), (2, 0)):
            c.set_option(A.OPT_SEARCH_IMPL, impl)
            c.set_option(A.OPT_SEARCH_CHUNK, chunk)
            rr = c.integer_search([10, 10], [1, M], [1, N], 30, 16)
            assert np.array_equal(rr["u"], r0["u"], equal_nan=True), (impl, chunk)
            assert np.array_equal(rr["v"], r0["v"], equal_nan=True), (impl, chunk)
        with pytest.raises(Exception):
            c.set_option(A.OPT_SLOW_WARPS, 3)
    finally:
        c.close()


@pytest.fixture(scope="module")
def hole():
    return synth.plate_with_hole(size=384, hole_r=60.0, peak=2.0, sin_amp=0.3, sin_wl=120.0)


def test_local_icgn_quadtree_masked_parity(ctx, hole):
    sc = hole
    M, N = sc.ref.shape
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(20, 370, 8.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    res = ctx.local_icgn(1, coords, U0, 24, 1e-3)
    ref = O.local_icgn(O.Frame(f, g, sc.mask, gx, gy), coords, U0, 24, 1e-3, variant=1)
    codes = set(np.unique(ref["conv"]).tolist())
    assert {-1, 102}.issubset(codes)  # regrowth mismatch and masked-out subsets occur
    assert np.mean(res["conv"] == ref["conv"]) >= 0.99
    assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
    assert np.array_equal(res["markHole"], ref["markHole"])
    both = _flag(res["conv"]) & _flag(ref["conv"])
    du = np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both]
    assert du.max() < UV_TOL
    m102 = ref["conv"] == 102
    assert np.array_equal(res["U"].reshape(-1, 2)[m102], U0.reshape(-1, 2)[m102])


def test_local_icgn_quadtree_masked_deformed_image(ctx, hole):
    # reference frame unmasked, deformed frame zeroed inside the hole (TemporalMatch's
    # gNormalized = ImgNormalized .* gMask): exact zeros in g start the per-iteration
    # g-region flood fill of funICGNQuadtree.m:170-182 on subsets without any f mask
    sc = hole
    M, N = sc.ref.shape
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N])
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N], mask=sc.mask)
    ctx.set_mask(None)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    assert np.sum(g == 0) > 1000
    xs = np.arange(24, 362, 7.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    res = ctx.local_icgn(1, coords, U0, 24, 1e-3)
    ref = O.local_icgn(O.Frame(f, g, None, gx, gy), coords, U0, 24, 1e-3, variant=1)
    assert np.mean(res["conv"] == ref["conv"]) >= 0.99
    assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
    both = _flag(res["conv"]) & _flag(ref["conv"])
    assert np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both].max() < UV_TOL


def test_subpb1_quadtree_parity(ctx, hole):
    sc = hole
    M, N = sc.ref.shape
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(20, 370, 10.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    n = len(coords)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    rng = np.random.default_rng(0)
    UOld = np.stack([tu, tv], 1).ravel() + rng.normal(0, 0.2, 2 * n)
    FOld = np.tile([0.005, 0.0, 0.0, -0.002], n)
    vdual = rng.normal(0, 0.05, 2 * n)
    wl = np.full((n, 2), 24, dtype=np.int32)
    res = ctx.subpb1(1, coords, UOld, FOld, vdual, 1e-3, 1e-3, winsize=24, winsize_list=wl)
    ref = O.subpb1(O.Frame(f, g, sc.mask, gx, gy), coords, UOld, FOld, vdual, 1e-3, 1e-3, winsize_list=wl, variant=1)
    assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
    assert np.mean(res["conv"] == ref["conv"]) >= 0.98
    both = _flag(res["conv"]) & _flag(ref["conv"])
    assert both.sum() > 0.5 * n
    du = np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both]
    assert du.max() < UV_TOL
    err = ref["conv"] == 0
    assert np.all(np.isnan(res["U"].reshape(-1, 2)[err]))


def test_subpb1_quadtree_mixed_windows_and_slow_subsets(A, ctx, hole):
    # per-subset windows 16 / 24 / 32 (queue 0 holds only the nominal size; the others are
    # unmasked queue-1 subsets solved by the warp-group passes); with an iteration cap of 1
    # every subset needing more than one iteration restarts in the multi-warp pass
    sc = hole
    M, N = sc.ref.shape
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(24, 366, 9.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    n = len(coords)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    rng = np.random.default_rng(3)
    UOld = np.stack([tu, tv], 1).ravel() + rng.normal(0, 0.2, 2 * n)
    FOld = np.tile([0.004, 0.0, 0.0, -0.002], n)
    vdual = rng.normal(0, 0.05, 2 * n)
    wsz = rng.choice([16, 24, 32], n).astype(np.int32)
    wl = np.stack([wsz, wsz], 1)
    ref = O.subpb1(O.Frame(f, g, sc.mask, gx, gy), coords, UOld, FOld, vdual, 1e-3, 1e-3, winsize_list=wl,
                   variant=1)
    assert np.sum(ref["conv"] > 1) > n // 4
    try:
        for cap in (16, 1):
            ctx.set_iteration_cap(cap)
            res = ctx.subpb1(1, coords, UOld, FOld, vdual, 1e-3, 1e-3, winsize=24, winsize_list=wl)
            assert np.mean(res["conv"] == ref["conv"]) >= 0.98, cap
            assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE, cap
            both = _flag(res["conv"]) & _flag(ref["conv"])
            assert np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both].max() < UV_TOL, cap
            assert np.array_equal(np.isnan(res["U"]), np.isnan(ref["U"])), cap
    finally:
        ctx.set_iteration_cap(A.DEFAULT_ITERATION_CAP)


def test_local_icgn_slow_subsets_restart(A, ctx, affine):
    # with an iteration cap of 1 every subset that needs a second iteration is restarted by
    # the multi-warp pass; codes and displacements still match the oracle
    _load_raw(ctx, affine)
    M, N = affine.ref.shape
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0 = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
    ref = O.local_icgn(O.Frame(f, g, None, gx, gy), coords, U0, 30, 1e-3, variant=0)
    assert np.sum(ref["conv"] > 1) > len(coords) // 2
    try:
        ctx.set_iteration_cap(1)
        ctx.set_option(A.OPT_SLOW_FP64, 1)
        res = ctx.local_icgn(0, coords, U0, 30, 1e-3)  # long trajectories re-solved in FP64
        ctx.set_option(A.OPT_SLOW_FP64, 0)
        for nw in (2, 4):  # the FP32 multi-warp pass instead
            ctx.set_option(A.OPT_SLOW_WARPS, nw)
            r32 = ctx.local_icgn(0, coords, U0, 30, 1e-3)
            assert np.mean(r32["conv"] == ref["conv"]) >= 0.98, nw
            assert np.mean(_flag(r32["conv"]) == _flag(ref["conv"])) >= FLAG_RATE, nw
            b32 = _flag(r32["conv"]) & _flag(ref["conv"])
            assert np.abs(r32["U"] - ref["U"]).reshape(-1, 2)[b32].max() < UV_TOL, nw
    finally:
        ctx.set_iteration_cap(A.DEFAULT_ITERATION_CAP)
        ctx.set_option(A.OPT_SLOW_FP64, 0)
        ctx.set_option(A.OPT_SLOW_WARPS, 2)
    assert np.array_equal(res["conv"], ref["conv"])
    ok = _flag(ref["conv"])
    assert np.abs(res["U"] - ref["U"]).reshape(-1, 2)[ok].max() < 1e-6
    with pytest.raises(Exception):
        ctx.set_iteration_cap(0)


def test_subpb1_uniform_parity(ctx, affine):
    sc = affine
    _load_raw(ctx, sc)
    M, N = sc.ref.shape
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    xs = np.arange(40, 480, 24.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    n = len(coords)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    loc = O.local_icgn(O.Frame(f, g, None, gx, gy), coords, U0, 30, 1e-3, variant=0)
    HPar = loc["H"]
    vdual = np.zeros(2 * n)
    res = ctx.subpb1(0, coords, loc["U"], loc["F"], vdual, 1e-3, 1e-3, winsize=30, HPar=HPar)
    ref = O.subpb1(O.Frame(f, g, None, gx, gy), coords, loc["U"], loc["F"], vdual, 1e-3, 1e-3, winsize=30,
                   HPar=HPar, variant=0)
    assert np.mean(_flag(res["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
    both = _flag(res["conv"]) & _flag(ref["conv"])
    assert np.abs(res["U"] - ref["U"]).reshape(-1, 2)[both].max() < UV_TOL


def test_epipolar_znssd_parity(ctx, affine):
    sc = affine
    _load_raw(ctx, sc)
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    rng = np.random.default_rng(3)
    pts = np.round(rng.uniform(40, 470, (200, 2)))
    z = ctx.epipolar_icgn(pts, 30, 1e-3)
    zo, _ = O.epipolar_icgn(O.Frame(f, g, None, gx, gy), pts, 30, 1e-3)
    ok = np.isfinite(zo)
    assert np.array_equal(np.isfinite(z), ok)
    assert np.max(np.abs(z[ok] - zo[ok])) < 1e-4


def test_triangulation_parity(ctx):
    st = synth.stereo_pair(size=256, f=500.0)
    rng = np.random.default_rng(8)
    pts = rng.uniform(30, 220, (2000, 2))
    tr = synth.stereo_truth(st, pts)
    pairs = np.hstack([pts, tr["right0"]]) + rng.normal(0, 0.02, (2000, 4))
    pairs[5, 1] = np.nan
    xo, eo = O.triangulate(pairs, st.KL, st.KR, st.R_rl, st.T_rl)
    xg, eg = ctx.triangulate(pairs, st.KL, st.KR, st.R_rl, st.T_rl)
    ok = np.isfinite(xo[:, 0])
    assert np.array_equal(np.isfinite(xg[:, 0]), ok) and not ok[5]
    assert np.max(np.abs(xg[ok] - xo[ok]) / np.abs(xo[ok]).max(axis=1, keepdims=True)) < 1e-5
    assert np.max(np.abs(eg[ok] - eo[ok])) < 1e-6


def test_device_pointer_path_matches_host_path(A, ctx, affine):
    import torch

    sc = affine
    _load_raw(ctx, sc)
    M, N = sc.ref.shape
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0 = np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1).ravel()
    host = ctx.local_icgn(1, coords, U0, 30, 1e-3)
    n = len(coords)
    dev = torch.device("cuda:0")
    side = torch.cuda.Stream(dev)
    with torch.cuda.stream(side):
        out = {"U": torch.empty(2 * n, dtype=torch.float64, device=dev),
               "F": torch.empty(4 * n, dtype=torch.float64, device=dev),
               "H": torch.empty(21 * n, dtype=torch.float64, device=dev),
               "conv": torch.empty(n, dtype=torch.int32, device=dev),
               "mark": torch.empty(n, dtype=torch.uint8, device=dev)}
        # MATLAB n x 2 column-major memory == a (2, n) row-major tensor
        c_t = torch.from_numpy(np.ascontiguousarray(coords.T)).to(dev)
        u_t = torch.from_numpy(U0).to(dev)
        ctx.set_stream(side.cuda_stream)
        ctx.local_icgn(1, c_t, u_t, 30, 1e-3, out=out)
    side.synchronize()
    ctx.set_stream(None)
    assert np.array_equal(out["conv"].cpu().numpy(), host["conv"])
    assert np.array_equal(out["U"].cpu().numpy(), host["U"], equal_nan=True)
    with pytest.raises(A.AldicError):  # a flat tensor carries no row count
        ctx.local_icgn(1, c_t.view(-1), u_t, 30, 1e-3, out=out)
    with pytest.raises(A.AldicError):  # too small an output is refused before launch
        small = dict(out, U=torch.empty(3, dtype=torch.float64, device=dev))
        ctx.local_icgn(1, c_t, u_t, 30, 1e-3, out=small)


def test_pinned_host_outputs_and_threaded_contexts(A, ctx, affine):
    """Results written in place into pinned host arrays (out=) equal the returned arrays,
    and three contexts driven from three host threads give the serial results."""
    import threading

    import torch

    sc = affine
    M, N = sc.ref.shape
    _load_raw(ctx, sc)
    ref_grid = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    nY, nX = ref_grid["u"].shape
    coords = np.stack([ref_grid["x"].T.ravel(order="F"), ref_grid["y"].T.ravel(order="F")], 1)
    U0 = np.stack([ref_grid["u"].T.ravel(order="F"), ref_grid["v"].T.ravel(order="F")], 1).ravel()
    ref_icgn = ctx.local_icgn(1, coords, U0, 30, 1e-3)
    n = len(coords)

    def pinned(k, dtype=np.float64):
        return torch.empty(k, dtype=getattr(torch, np.dtype(dtype).name), pin_memory=True).numpy()

    ctxs = [A.Context(0) for _ in range(3)]
    outs = [{**{nm: pinned(nX * nY) for nm in ("x", "y", "u", "v", "phi")}, "U": pinned(2 * n),
             "F": pinned(4 * n), "H": pinned(21 * n), "conv": pinned(n, np.int32)} for _ in range(3)]
    errors = []

    def run(i):
        try:
            c, o = ctxs[i], outs[i]
            c.load_image_raw(0, sc.ref, [1, M], [1, N])
            c.load_image_raw(1, sc.deff, [1, M], [1, N])
            c.compute_gradients()
            for _ in range(3):
                assert c.integer_search([10, 10], [1, M], [1, N], 30, 16, out=o) is o
                assert c.local_icgn(1, coords, U0, 30, 1e-3, out=o) is o
        except Exception as e:  # reported on the main thread
            errors.append(e)

    th = [threading.Thread(target=run, args=(i,)) for i in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in ctxs:
        c.close()
    assert not errors, errors
    for o in outs:
        for nm in ("u", "v", "phi"):
            assert np.array_equal(o[nm].reshape((nY, nX), order="F"), ref_grid[nm], equal_nan=True), nm
        assert np.array_equal(o["conv"], ref_icgn["conv"])
        assert np.array_equal(o["U"], ref_icgn["U"], equal_nan=True)
        assert np.array_equal(o["H"], ref_icgn["H"].ravel(order="F"), equal_nan=True)
    with pytest.raises(A.AldicError):  # a float32 array would take the results into a temporary
        ctx.local_icgn(1, coords, U0, 30, 1e-3, out=dict(outs[0], U=np.empty(2 * n, np.float32)))


def test_inpaint_nans_and_init_parity(A, ctx):
    """inpaint_nans(., 4) and Init(., 0) against the oracle's spring-system solve: scattered
    NaNs, a block hole, border runs, a whole edge column; unchanged finite entries; the
    device-tensor path; a grid without NaN; an all-NaN grid (no finite neighbour -> 0)."""
    import torch

    rng = np.random.default_rng(11)
    for m, n in ((40, 55), (200, 200), (7, 3)):
        G = rng.normal(size=(m, n)) * 3.0
        G[rng.random(G.shape) < 0.1] = np.nan
        G[m // 4:m // 2, n // 3:n // 2] = np.nan
        G[0, : n // 2] = np.nan
        G[:, -1] = np.nan
        ref = O.inpaint_nans4(G)
        got, info = ctx.inpaint_nans(G, info=True)
        assert info[0] == int(np.isnan(G).sum()) and info[2] == 1, info
        assert np.array_equal(got[np.isfinite(G)], G[np.isfinite(G)])
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-10 * scale, (m, n)
        # device path, in place ((n, m) row-major tensor == column-major m x n)
        t = torch.from_numpy(np.ascontiguousarray(G.T)).cuda()
        ctx.inpaint_nans(t)
        torch.cuda.synchronize()
        assert np.abs(t.cpu().numpy().T - ref).max() <= 1e-10 * scale
    clean = rng.normal(size=(9, 12))
    assert np.array_equal(ctx.inpaint_nans(clean), clean)
    assert np.array_equal(ctx.inpaint_nans(np.full((4, 5), np.nan)), np.zeros((4, 5)))
    # Init: the search grids of a real search, with holes punched in
    sc = synth.temporal_affine()
    _load_raw(ctx, sc)
    M, N = sc.ref.shape
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    u, v = r["u"].copy(), r["v"].copy()
    u[rng.random(u.shape) < 0.2] = np.nan
    v[np.isnan(u)] = np.nan
    u_in, v_in = u.copy(), v.copy()
    U0 = ctx.init_u0(u, v)
    ref = O.init_u0(u, v)
    assert np.abs(U0 - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.array_equal(u, u_in, equal_nan=True) and np.array_equal(v, v_in, equal_nan=True)
    assert np.array_equal(A.Init(u, v, ctx=ctx), U0)
    # index 1: the spring outlier passes, with planted outliers (same NaN marks as the oracle,
    # whose operations are rounded one by one like the device's)
    uo, vo = r["u"].copy(), r["v"].copy()
    uo[4, 6] += 9.0
    vo[10, 3] -= 7.0
    uo[rng.random(uo.shape) < 0.05] = np.nan
    U1 = ctx.init_u0(uo, vo, index=1)
    ref1 = O.init_u0(uo, vo, index=1)
    assert np.abs(U1 - ref1).max() <= 1e-9 * max(1.0, np.abs(ref1).max())
    assert abs(U1[0::2].reshape(uo.shape)[4, 6] - r["u"][4, 6]) < 1.0  # the outlier is gone


def test_undistort_and_reconstruction_parity(A, ctx):
    """funUndistortPoints against the oracle's restatement and the forward lens model; the
    reconstruction driver with distortion recovers the points triangulated without it."""
    K = np.array([[4000.0, 0.5, 1024.5], [0, 4010.0, 1000.2], [0, 0, 1]])
    rng = np.random.default_rng(2)
    P = rng.uniform(1, 2048, (3000, 2))
    P[7] = np.nan
    for rad, tan in (([-0.12, 0.05, -0.01], [1e-3, -5e-4]), ([0.08, -0.02], None), ([0.0, 0.0], None)):
        got = ctx.undistort_points(P, K, rad, tan)
        ref = O.undistort_points(P, K, rad, tan)
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        ok = np.isfinite(ref[:, 0])
        assert np.abs(got[ok] - ref[ok]).max() < 1e-9
        assert np.abs(O.distort_points(got[ok], K, rad, tan) - P[ok]).max() < 1e-9
    sc = synth.stereo_pair(seed=3, size=256, f=500.0)
    xy = rng.uniform(60, 200, (400, 2))
    tr = synth.stereo_truth(sc, xy)
    pairs = np.hstack([xy, tr["right0"]])
    cam = {"KL": sc.KL, "KR": sc.KR, "R": sc.R_rl, "T": sc.T_rl}
    plain, _ = A.stereoReconstruction_quadtree([pairs], cam, ctx=ctx)
    lens = dict(cam, radialL=[-0.05, 0.01], tangentialL=[2e-4, 1e-4], radialR=[0.04, 0.0, -0.002])
    dist_pairs = np.hstack([O.distort_points(pairs[:, :2], sc.KL, lens["radialL"], lens["tangentialL"]),
                            O.distort_points(pairs[:, 2:], sc.KR, lens["radialR"])])
    und = A.funUndistortPoints([dist_pairs], lens, ctx=ctx)[0]
    assert np.abs(und - pairs).max() < 1e-8
    lensed, _ = A.stereoReconstruction_quadtree([dist_pairs], lens, ctx=ctx)
    assert np.abs(lensed["Coordinates"][0] - plain["Coordinates"][0]).max() < 1e-6


def test_integer_search_quadtree_driver(A, ctx, affine):
    """IntegerSearchQuadtree: the distance from DICpara, the device search, mask -> NaN."""
    sc = affine
    M, N = sc.ref.shape
    mask = np.ones((M, N))
    mask[200:320, 150:260] = 0
    para = {"gridxyROIRange": {"gridx": [1, M], "gridy": [1, N]}, "winsize": 30, "winstepsize": 16,
            "TemporalSearchDistance": 10, "ImgRefMask": mask}
    para2, x0, y0, u, v, cc = A.IntegerSearchQuadtree(sc.ref, sc.deff, None, para, 2, ctx=ctx)
    xr, yr, ur, vr, _ = A.funIntegerSearch(sc.ref, sc.deff, [10, 10], [1, M], [1, N], 30, 16, ctx=ctx)
    hole = mask[np.floor(x0 + 0.5).astype(int) - 1, np.floor(y0 + 0.5).astype(int) - 1] == 0
    assert hole.sum() > 10 and (~hole).sum() > 100
    assert np.isnan(u[hole]).all() and np.isnan(v[hole]).all()
    # then funRemoveOutliers(u, v, cc, 0, 100), as the oracle restates it
    uo, vo, _ = O.remove_outliers(np.where(hole, np.nan, ur), np.where(hole, np.nan, vr), 100.0)
    assert np.array_equal(np.isnan(u), np.isnan(uo)) and np.array_equal(np.isnan(v), np.isnan(vo))
    assert np.nanmax(np.abs(u - uo)) < 1e-9 and np.nanmax(np.abs(v - vo)) < 1e-9
    assert list(para2["SizeOfFFTSearchRegion"]) == [10, 10]


def _outlier_grids(seed, m=40, n=35):
    rng = np.random.default_rng(seed)
    R, C = np.meshgrid(np.arange(m, dtype=float), np.arange(n, dtype=float), indexing="ij")
    u = np.round(3.37 + 0.02 * R - 0.01 * C + 0.3 * np.sin(R / 6.0), 3)
    v = np.round(-1.82 + 0.015 * C + 0.2 * np.cos(C / 5.0), 3)
    bad = rng.random((m, n)) < 0.03
    u[bad] += rng.choice([-1, 1], bad.sum()) * rng.uniform(15, 60, bad.sum())
    v[rng.random((m, n)) < 0.02] -= 30.0
    u[14:19, 9:15] = np.nan  # a mask hole (as IntegerSearchQuadtree leaves it)
    v[14:19, 9:15] = np.nan
    u[0, 0] = v[0, 0] = np.nan
    return u, v


@pytest.mark.parametrize("seed", [0, 1])
def test_remove_outliers_parity(A, ctx, seed):
    """funRemoveOutliers(u, v, cc, 0, 100): the removed entries bit-exact against the oracle
    (single-precision median test), the inpainted grids to 1e-9, the holes NaN again."""
    import torch

    u, v = _outlier_grids(seed)
    uo, vo, bad = O.remove_outliers(u, v, 100.0)
    ug, vg, info = ctx.remove_outliers(u, v, 100.0, info=True)
    assert info[0] == bad.size and bad.size > 5
    assert info[1] == int(np.isnan(u).sum()) and info[3] == 1
    assert np.array_equal(np.isnan(ug), np.isnan(uo)) and np.array_equal(np.isnan(vg), np.isnan(vo))
    assert np.nanmax(np.abs(ug - uo)) < 1e-9 and np.nanmax(np.abs(vg - vo)) < 1e-9
    # the driver form and the device-tensor form (in place) agree with the host form
    u2, v2, _ = A.funRemoveOutliers(u, v, {}, 0, 100, ctx=ctx)
    assert np.array_equal(u2, ug, equal_nan=True) and np.array_equal(v2, vg, equal_nan=True)
    tu = torch.from_numpy(np.ascontiguousarray(u.T)).cuda()
    tv = torch.from_numpy(np.ascontiguousarray(v.T)).cuda()
    ctx.remove_outliers(tu, tv, 100.0)
    torch.cuda.synchronize()
    assert np.array_equal(tu.cpu().numpy().T, ug, equal_nan=True)
    assert np.array_equal(tv.cpu().numpy().T, vg, equal_nan=True)


def test_remove_outliers_edges(A, ctx):
    """No NaN and no outlier: the grids come back unchanged; empty grids are a no-op; a zero
    threshold (the reference's prompt) is an error."""
    R, C = np.meshgrid(np.arange(12.0), np.arange(9.0), indexing="ij")
    u, v = 1.0 + 0.1 * R, 2.0 - 0.05 * C
    ug, vg, info = ctx.remove_outliers(u, v, 100.0, info=True)
    assert info == (0, 0, 0, 1) and np.array_equal(ug, u) and np.array_equal(vg, v)
    e = np.zeros((0, 4))
    assert ctx.remove_outliers(e, e)[0].shape == (0, 4)
    with pytest.raises(A.AldicError):
        ctx.remove_outliers(u, v, 0.0)
    with pytest.raises(A.AldicError):
        A.funRemoveOutliers(u, v, {}, 1, 100, ctx=ctx)


def test_launch_counter_and_errors(A, ctx):
    before = ctx.launches
    ctx.triangulate(np.zeros((4, 4)) + 1.0, np.eye(3), np.eye(3), np.eye(3), [1.0, 0, 0])
    assert ctx.launches > before
    with pytest.raises(A.AldicError):
        ctx.local_icgn(1, np.zeros((3, 2)), np.zeros(6), 1000, 1e-3)


@pytest.mark.parametrize("order,dirichlet", [(2, ()), (2, (4, 9, 17, 30)), (3, (2,))])
def test_subpb2_parity(A, ctx, order, dirichlet):
    """Subpb2Quadtree: the device's element assembly and preconditioned CG against the
    oracle's element-by-element assembly and direct solve, on a quadtree mesh with hanging
    nodes; the driver form with a DICmesh dict gives the same."""
    from test_subpb2_host import quadtree_mesh

    C, E = quadtree_mesh(7, {(1, 1), (2, 1), (4, 4), (5, 2)})
    n = C.shape[0]
    rng = np.random.default_rng(11 + order)
    U = 3.0 + rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    for beta in (1e-3 * 16 ** 2 * 1e-3, 1e-1 * 16 ** 2 * 1e-3):
        ref = O.subpb2_quadtree(C, E, order, beta, 1e-3, U, F, dirichlet=dirichlet)
        got, nfo = ctx.subpb2(C, E, order, beta, 1e-3, U, F, dirichlet=dirichlet or None, info=True)
        assert nfo[1] == 1 and nfo[0] > 0
        assert np.abs(got - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())
    mesh = {"coordinatesFEM": C, "elementsFEM": E, "dirichlet": list(dirichlet), "neumann": []}
    drv = A.Subpb2Quadtree(mesh, order, beta, 1e-3, U, F, np.zeros(4 * n), np.zeros(2 * n), 0.0, 16, 0, ctx=ctx)
    assert np.array_equal(drv, got)


def test_subpb2_device_tensors_and_errors(A, ctx):
    """Device-resident inputs and output give the host result; bad tables and parameters
    are errors, not faults."""
    import torch

    from test_subpb2_host import quadtree_mesh

    C, E = quadtree_mesh(5, {(1, 2), (3, 3)})
    n = C.shape[0]
    rng = np.random.default_rng(3)
    U = rng.standard_normal(2 * n)
    F = 0.02 * rng.standard_normal(4 * n)
    host = ctx.subpb2(C, E, 2, 0.0256, 1e-3, U, F)
    dev = torch.device("cuda:0")
    tC = torch.from_numpy(np.ascontiguousarray(C.T)).to(dev)
    tE = torch.from_numpy(np.ascontiguousarray(E.T.astype(np.int32))).to(dev)
    tU, tF = torch.from_numpy(U).to(dev), torch.from_numpy(F).to(dev)
    out = torch.empty(2 * n, dtype=torch.float64, device=dev)
    ctx.subpb2(tC, tE, 2, 0.0256, 1e-3, tU, tF, out=out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)
    # the resident mesh gives the same; a node count that does not match it is an error
    ctx.subpb2_set_mesh(n, E)
    assert np.array_equal(ctx.subpb2(C, None, 2, 0.0256, 1e-3, U, F), host)
    with pytest.raises(A.AldicError):
        ctx.subpb2(C[:-1], None, 2, 0.0256, 1e-3, U[:-2], F[:-4])
    bad = E.copy()
    bad[0, 0] = 0
    with pytest.raises(A.AldicError):
        ctx.subpb2(C, bad, 2, 0.0256, 1e-3, U, F)
    bad = E.copy()
    bad[1, 5] = n + 3
    with pytest.raises(A.AldicError):
        ctx.subpb2(C, bad, 2, 0.0256, 1e-3, U, F)
    with pytest.raises(A.AldicError):
        ctx.subpb2(C, E, 6, 0.0256, 1e-3, U, F)
    with pytest.raises(A.AldicError):
        ctx.subpb2(C, E, 2, 0.0, 0.0, U, F)
    with pytest.raises(A.AldicError):
        ctx.subpb2(C, E, 2, 0.0256, 1e-3, U, F, dirichlet=[n + 1])
    with pytest.raises(A.AldicError):
        A.Subpb2Quadtree({"coordinatesFEM": C, "elementsFEM": E, "neumann": [[1, 2, 0, 1]]}, 2, 0.1, 1e-3, U, F,
                         ctx=ctx)



def test_local_icgn_quadtree_driver_fill(A, ctx, hole):
    """LocalICGNQuadtree as the reference returns it: the device loop, the bad-point rules,
    then the natural-neighbour fill per mask region and over the mesh; bad nodes (inside
    the hole, failed subsets) filled, good nodes untouched."""
    from aldic_b200.fill import fill_quadtree

    sc = hole
    ctx.load_image_raw(0, sc.ref, [1, sc.ref.shape[0]], [1, sc.ref.shape[1]], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, sc.ref.shape[0]], [1, sc.ref.shape[1]])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    Df = {"DfDx": ctx.get_state(2), "DfDy": ctx.get_state(3), "ImgRefMask": sc.mask}
    xs = np.arange(24, 366, 12.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    U, F, H, t, conv, num, mark = A.LocalICGNQuadtree(U0, coords, Df, f, g, {"winsize": 24}, tol=1e-3, ctx=ctx)
    Un, _, _, _, conv2, num2, _ = A.LocalICGNQuadtree(U0, coords, Df, f, g, {"winsize": 24}, tol=1e-3, ctx=ctx,
                                                      fill=False)
    bad = np.isnan(Un[0::2])
    assert num == num2 and bad.sum() > 10 and np.array_equal(conv, conv2)
    assert np.isfinite(U).all()
    assert np.array_equal(U.reshape(-1, 2)[~bad], Un.reshape(-1, 2)[~bad])
    assert np.array_equal(U, fill_quadtree(Un, coords, sc.mask))


def test_quadtree_aldic_frame_parity(A, ctx):
    """A reduced form of the quadtree ALDIC frame: a plate with a hole and an edge notch, the
    GenerateQuadtreeMesh mesh refined at the mask edges, LocalICGNQuadtree, then two ADMM
    rounds of Subpb2Quadtree + Subpb1Quadtree (func/TemporalMatch_quadtree_ST1.m:248-380);
    every device step against the oracle on the same inputs (the device's results of the
    step before): codes, flags and u/v within the bar, the global steps to 1e-8 px."""
    sc = synth.plate_with_hole(seed=5, size=512, hole_r=75.0, peak=2.0, sin_amp=0.3, sin_wl=100.0)
    M, N = sc.ref.shape
    w, st, mu, tol = 24, 8, 1e-3, 1e-3
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    f, g = ctx.get_state(0), ctx.get_state(1)
    gx, gy = ctx.get_state(2), ctx.get_state(3)
    frame = O.Frame(f, g, sc.mask, gx, gy)
    xl = np.arange(1, M - w - st + 1, st) + w / 2.0
    yl = np.arange(1, N - w - st + 1, st) + w / 2.0
    X, Y = np.meshgrid(xl, yl, indexing="ij")
    mesh0 = A.MeshSetUp(X.T, Y.T, {"winstepsize": st, "ImgSize": [M, N]})
    mesh0["elementMinSize"] = 4
    qmesh, _, _ = A.GenerateQuadtreeMesh(np.zeros(2 * X.size), None, sc.mask, mesh0, {"winstepsize": st, "winsize": w})
    coords, E, dirichlet = qmesh["coordinatesFEM"], qmesh["elementsFEM"], list(qmesh["dirichlet"])
    n = coords.shape[0]
    assert n > X.size and E.shape[1] == 8 and np.any(E[:, 4:] > 0)  # refined, with hanging nodes
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()

    def agree(got, ref):
        fl = _flag(got["conv"]) & _flag(ref["conv"])
        assert np.mean(_flag(got["conv"]) == _flag(ref["conv"])) >= FLAG_RATE
        assert np.mean(got["conv"] == ref["conv"]) >= 0.99
        assert fl.sum() > 0.5 * n
        assert np.abs(got["U"] - ref["U"]).reshape(-1, 2)[fl].max() < UV_TOL

    loc = ctx.local_icgn(1, coords, U0, w, tol)
    lref = O.local_icgn(frame, coords, U0, w, tol, variant=1, nthreads=8)
    agree(loc, lref)
    assert np.array_equal(loc["markHole"], lref["markHole"])
    U1 = np.where(np.isnan(loc["U"]), U0, loc["U"])
    F1 = np.nan_to_num(loc["F"])
    hole = np.repeat(loc["markHole"].astype(bool), 2)
    wl = np.full((n, 2), w, dtype=np.int32)
    beta = 1e-2 * st ** 2 * mu
    for _ in range(2):
        U2 = ctx.subpb2(coords, E, 2, beta, mu, U1, F1, dirichlet=dirichlet)
        ref2 = O.subpb2_quadtree(coords, E, 2, beta, mu, U1, F1, dirichlet=dirichlet)
        assert np.abs(U2 - ref2).max() < 1e-8
        U2 = np.where(hole, U1, U2)
        vdual = U2 - U1
        s1 = ctx.subpb1(1, coords, U2, F1, vdual, mu, tol, winsize=w, winsize_list=wl)
        agree(s1, O.subpb1(frame, coords, U2, F1, vdual, mu, tol, winsize_list=wl, variant=1, nthreads=8))
        U1 = np.where(np.isnan(s1["U"]), U2, s1["U"])
