"""The allocation-free IC-GN entry point (aldic_local_icgn_noalloc).

Callers that own every device allocation themselves (a MEX passing gpuArray buffers, an
application with its own pool or a fixed budget) can pass inputs and outputs but cannot
let the library allocate; this entry point keeps its work queue in a fixed device array.
The test calls it through the C ABI, twice in a row on different batches, and checks
each result against the context-based aldic_local_icgn on the same device inputs,
within the parity tolerances of the other GPU tests.  The file sorts last so that a run
stopping at the first failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from aldic_b200 import synth

pytestmark = pytest.mark.gpu

UV_TOL = 1e-3


def _flag(conv):
    return (conv > 0) & (conv < 100)


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
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel(order="F")).astype(np.float32)).to(dev)
    ref, deff, gx, gy = (f32(ctx.get_state(k)) for k in range(4))
    r = ctx.integer_search([10, 10], [1, M], [1, N], 30, 16)
    coords_all = np.stack([r["x"].T.ravel(order="F"), r["y"].T.ravel(order="F")], 1)
    U0_all = np.nan_to_num(np.stack([r["u"].T.ravel(order="F"), r["v"].T.ravel(order="F")], 1)).ravel()
    stream = torch.cuda.Stream(dev)
    batches = [(1, slice(0, 600)), (0, slice(300, 900))]  # two calls in a row, different batches
    for variant, sl in batches:
        coords = coords_all[sl]
        U0 = U0_all[2 * sl.start:2 * sl.stop]
        n = coords.shape[0]
        want = ctx.local_icgn(variant, coords, U0, 30, 1e-3)
        c_t = torch.from_numpy(np.ascontiguousarray(coords.T)).to(dev)
        u0_t = torch.from_numpy(np.ascontiguousarray(U0)).to(dev)
        U = torch.full((2 * n,), -7.0, dtype=torch.float64, device=dev)
        F = torch.full((4 * n,), -7.0, dtype=torch.float64, device=dev)
        H = torch.full((21 * n,), -7.0, dtype=torch.float64, device=dev)
        conv = torch.full((n,), -7, dtype=torch.int32, device=dev)
        mark = torch.zeros(n, dtype=torch.uint8, device=dev)
        p = lambda t: C.c_void_p(t.data_ptr())
        torch.cuda.synchronize(dev)
        rc = lib.aldic_local_icgn_noalloc(variant, p(ref), p(deff), None, p(gx), p(gy), M, N, n, p(c_t), p(u0_t),
                                          30, 1e-3, p(U), p(F), p(H), p(conv), p(mark),
                                          C.c_void_p(stream.cuda_stream))
        assert rc == 0
        stream.synchronize()
        got_conv = conv.cpu().numpy()
        assert np.mean(_flag(got_conv) == _flag(want["conv"])) >= 0.999
        both = _flag(got_conv) & _flag(want["conv"])
        assert both.sum() > 0.8 * n
        dU = np.abs(U.cpu().numpy() - want["U"]).reshape(-1, 2)[both]
        assert dU.max() <= UV_TOL
        assert np.array_equal(np.isnan(U.cpu().numpy()), np.isnan(want["U"]))
    ctx.close()


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
