"""The allocation-free IC-GN entry point (aldic_local_icgn_noalloc).

Callers that own every device allocation themselves (a MEX passing gpuArray buffers, an
application with its own pool or a fixed budget) can pass inputs and outputs but cannot
let the library allocate; this entry point keeps its work queue in a fixed device array.
The tests call it through the C ABI, twice in a row, and check U, F, H, the codes and
markHole against the context-based aldic_local_icgn on the same device inputs (itself
checked against the FP64 oracle by the parity tests), within the parity tolerances of the
other GPU tests: an unmasked affine field (both variants) and a masked plate with a hole.  The file sorts last so that a run
stopping at the first failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from aldic_b200 import synth

pytestmark = pytest.mark.gpu

UV_TOL = 1e-3  # the parity tolerances of the other GPU tests
F_TOL = 1e-4
H_REL_TOL = 1e-5


def _f32(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F")).astype(np.float32)).to(dev)


def _flag(conv):
    return (conv > 0) & (conv < 100)


def _call(lib, dev, stream, variant, ref, deff, mask, gx, gy, M, N, coords, U0, w):
    import torch

    n = coords.shape[0]
    c_t = torch.from_numpy(np.ascontiguousarray(coords.T)).to(dev)
    u0_t = torch.from_numpy(np.ascontiguousarray(U0)).to(dev)
    out = {"U": torch.full((2 * n,), -7.0, dtype=torch.float64, device=dev),
           "F": torch.full((4 * n,), -7.0, dtype=torch.float64, device=dev),
           "H": torch.full((21 * n,), -7.0, dtype=torch.float64, device=dev),
           "conv": torch.full((n,), -7, dtype=torch.int32, device=dev),
           "markHole": torch.full((n,), 9, dtype=torch.uint8, device=dev)}
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    torch.cuda.synchronize(dev)
    rc = lib.aldic_local_icgn_noalloc(variant, p(ref), p(deff), p(mask), p(gx), p(gy), M, N, n, p(c_t), p(u0_t),
                                      w, 1e-3, p(out["U"]), p(out["F"]), p(out["H"]), p(out["conv"]),
                                      p(out["markHole"]), C.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["H"] = res["H"].reshape(21, n).T  # n x 21 column-major, as the context path returns it
    return res


def _compare(got, want, n, quad):
    assert np.mean(_flag(got["conv"]) == _flag(want["conv"])) >= 0.999
    assert np.mean(got["conv"] == want["conv"]) >= 0.99
    both = _flag(got["conv"]) & _flag(want["conv"])
    assert both.sum() > 0.5 * n
    dU = np.abs(got["U"] - want["U"]).reshape(-1, 2)[both]
    assert dU.max() <= UV_TOL
    dF = np.abs(got["F"] - want["F"]).reshape(-1, 4)[both]
    assert dF.max() <= F_TOL
    Hw = want["H"][both]
    scale = np.abs(Hw).max(axis=1, keepdims=True)
    assert np.max(np.abs(got["H"][both] - Hw) / scale) <= H_REL_TOL
    assert np.array_equal(np.isnan(got["U"]), np.isnan(want["U"]))
    if quad:
        assert np.array_equal(got["markHole"], want["markHole"])


def test_noalloc_matches_context_path_twice():
    import torch

    import aldic_b200 as A

    lib = A.load_library()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    sc = synth.temporal_affine()
    M, N = sc.ref.shape
    ctx = A.Context(0)
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N])
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.compute_gradients()
    # the context's FP32 device state, handed over as caller-owned device buffers
    ref, deff, gx, gy = (_f32(ctx.get_state(k), dev) for k in range(4))
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords_all = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0_all = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
    stream = torch.cuda.Stream(dev)
    batches = [(1, slice(0, 600)), (0, slice(300, 900))]  # two calls in a row, different batches
    for variant, sl in batches:
        coords = coords_all[sl]
        U0 = U0_all[2 * sl.start:2 * sl.stop]
        want = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
        got = _call(lib, dev, stream, variant, ref, deff, None, gx, gy, M, N, coords, U0, 30)
        _compare(got, want, coords.shape[0], variant == 1)
    ctx.close()


def test_noalloc_masked_quadtree_batch_matches_context_path():
    # a plate with a hole: enlarged windows, masked subsets solved by the general kernel,
    # codes -1 / 102 and markHole, with the mask handed over as a caller-owned u8 array
    import torch

    import aldic_b200 as A

    lib = A.load_library()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    sc = synth.plate_with_hole(size=384, hole_r=60.0, peak=2.0, sin_amp=0.3, sin_wl=120.0)
    M, N = sc.ref.shape
    ctx = A.Context(0)
    ctx.load_image_raw(0, sc.ref, [1, M], [1, N], mask=sc.mask)
    ctx.load_image_raw(1, sc.deff, [1, M], [1, N])
    ctx.set_mask(sc.mask)
    ctx.compute_gradients()
    ref, deff, gx, gy = (_f32(ctx.get_state(k), dev) for k in range(4))
    mask = torch.from_numpy(np.ascontiguousarray((sc.mask != 0).ravel(order="F")).astype(np.uint8)).to(dev)
    xs = np.arange(20, 370, 8.0)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()
    want = ctx.local_icgn(1, coords, U0, 24, 1e-3)
    assert {-1, 102}.issubset(set(np.unique(want["conv"]).tolist()))
    assert want["markHole"].sum() > 0
    stream = torch.cuda.Stream(dev)
    for _ in range(2):  # twice in a row: the shared array keeps nothing that matters
        got = _call(lib, dev, stream, 1, ref, deff, mask, gx, gy, M, N, coords, U0, 24)
        _compare(got, want, coords.shape[0], True)
    ctx.close()


def test_noalloc_refuses_memory_of_another_device():
    import torch

    import aldic_b200 as A

    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU")
    lib = A.load_library()
    torch.cuda.set_device(0)
    here = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    there = torch.zeros(64, dtype=torch.float64, device="cuda:1")
    p, q = C.c_void_p(here.data_ptr()), C.c_void_p(there.data_ptr())
    rc = lib.aldic_local_icgn_noalloc(1, q, p, None, p, p, 64, 64, 4, p, p, 30, 1e-3, p, p, None, p, None, None)
    assert rc == 1  # ALDIC_ERR_ARG: the reference image lives on another GPU


def test_noalloc_rejects_batches_beyond_the_fixed_queue():
    import torch

    import aldic_b200 as A

    lib = A.load_library()
    dev = torch.device("cuda:0")
    big = 65536 + 1
    t = torch.zeros(8, dtype=torch.float64, device=dev)
    p = C.c_void_p(t.data_ptr())
    rc = lib.aldic_local_icgn_noalloc(1, p, p, None, p, p, 64, 64, big, p, p, 30, 1e-3, p, p, None, p, None, None)
    assert rc == 1  # ALDIC_ERR_ARG, nothing queued
    host = np.zeros(8)
    rc = lib.aldic_local_icgn_noalloc(1, C.c_void_p(host.ctypes.data), p, None, p, p, 64, 64, 4, p, p, 30, 1e-3, p,
                                      p, None, p, None, None)
    assert rc == 1  # host memory is refused: every array must be device memory
