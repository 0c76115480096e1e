"""Host-side mirror of the reference's MATLAB interface for the per-subset hot path,
running on the B200 through the C ABI of libaldic_b200.so.

Function names, argument meaning, array layouts and per-subset status codes follow the
reference (func/, func_quadtree/): images are column-major M x N (numpy order='F', dim 1
= image x), coordinates 1-based, U interleaved [u1 v1 ...], F interleaved
[F11 F21 F12 F22 ...], HtempPar n x 21, ConvItPerEle codes (iterations / 101 / 102 / 103
/ -1).

Arrays may be numpy (host) or CUDA torch tensors (device); device arrays keep the call
asynchronous on the context's stream.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import fill as _fill
from . import smooth as _smooth
from . import _lib
from ._lib import AldicError

__all__ = [
    "Context", "default_context", "funNormalizeImg", "funImgGradient", "ba_interp2_spline", "funIntegerSearch",
    "LocalICGN", "LocalICGNQuadtree", "Subpb1", "Subpb1Quadtree", "epipolar_ICGN1",
    "stereoReconstruction_quadtree", "bad_points_local", "bad_points_subpb1", "Init", "funUndistortPoints",
    "IntegerSearchQuadtree", "MeshSetUp", "funRemoveOutliers", "Subpb2Quadtree", "GenerateQuadtreeMesh",
    "StereoMatch_STAQ", "ALDICFrameQuadtree", "subpb2_beta", "organizeMatchedPairds_quadtree_ST1",
    "TemporalMatch_quadtree_ST1",
]


def _is_torch(x):
    return hasattr(x, "data_ptr") and hasattr(x, "is_cuda")


class _Keep:
    """Holds converted numpy buffers alive for the duration of a call."""

    def __init__(self):
        self.items = []

    def ptr(self, x, dtype, order="F", numel=None):
        if x is None:
            return None
        if _is_torch(x):
            if not x.is_cuda or not x.is_contiguous():
                raise AldicError("device arrays must be contiguous CUDA tensors")
            want = str(np.dtype(dtype))
            if str(x.dtype).replace("torch.", "") != want:
                raise AldicError(f"device array has dtype {x.dtype}, expected {want}")
            if numel is not None and x.numel() < numel:
                raise AldicError(f"device array holds {x.numel()} elements, {numel} required")
            return C.c_void_p(x.data_ptr())
        a = np.asarray(x, dtype=dtype)
        a = np.ascontiguousarray(a.ravel(order=order)) if a.ndim > 1 else np.ascontiguousarray(a)
        self.items.append(a)
        return C.c_void_p(a.ctypes.data)

    def dst(self, x, dtype, numel):
        """An output the library writes in place: a CUDA tensor, or a writeable contiguous
        host numpy array of exactly `dtype` (in pinned host memory the device->host copy is
        a direct DMA).  Anything that would need a conversion is refused, since the results
        would land in a temporary."""
        if x is None:
            return None
        if _is_torch(x):
            return self.ptr(x, dtype, numel=numel)
        ok = isinstance(x, np.ndarray) and x.dtype == np.dtype(dtype) and x.flags.writeable and (
            x.flags.c_contiguous or x.flags.f_contiguous)
        if not ok:
            raise AldicError(f"outputs must be CUDA tensors or writeable contiguous {np.dtype(dtype)} numpy arrays")
        if x.size < numel:
            raise AldicError(f"output array holds {x.size} elements, {numel} required")
        return C.c_void_p(x.ctypes.data)

    def out(self, n, dtype):
        a = np.empty(n, dtype=dtype)
        self.items.append(a)
        return a, C.c_void_p(a.ctypes.data)


def _count(x, per_row):
    """Number of rows of an n x per_row MATLAB array: numpy (n, per_row), or a CUDA tensor
    of shape (per_row, n) (the same column-major memory)."""
    if _is_torch(x):
        if x.dim() != 2 or x.shape[0] != per_row:
            raise AldicError(f"device arrays of n x {per_row} MATLAB data are passed as ({per_row}, n) tensors")
        return int(x.shape[1])
    a = np.asarray(x)
    if a.ndim != 2 or a.shape[1] != per_row:
        raise AldicError(f"expected an n x {per_row} array, got shape {a.shape}")
    return int(a.shape[0])


def _img_shape(img, shape):
    """(M, N) of a column-major image: numpy arrays carry it; CUDA tensors need shape=."""
    if _is_torch(img):
        if shape is None or img.numel() != shape[0] * shape[1]:
            raise AldicError("device images need shape=(M, N) matching their element count")
        return int(shape[0]), int(shape[1])
    return img.shape


def _np_dtype_code(a):
    dt = a.dtype if hasattr(a, "dtype") else np.asarray(a).dtype
    name = str(dt).replace("torch.", "")
    return {"uint8": _lib.U8, "uint16": _lib.U16, "float32": _lib.F32, "float64": _lib.F64}[name]


class Context:
    """One device context: a CUDA stream, the resident frame (REF/DEF images, mask,
    gradients) and the scratch buffers of the batched solvers."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.aldic_create(C.byref(h), int(device))
        if rc != _lib.ALDIC_OK:
            raise AldicError(f"aldic_create(device={device}) failed with code {rc} (no usable CUDA device?)")
        self.h = h
        self.device = device
        self.M = self.N = None
        self._sp2_nel = -1  # elements of the resident global-step mesh (none yet)

    def close(self):
        if getattr(self, "h", None):
            self.lib.aldic_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != _lib.ALDIC_OK:
            msg = self.lib.aldic_last_error(self.h)
            raise AldicError(f"{what}: code {rc}: {msg.decode() if msg else ''}")

    # ------------------------------------------------------------------ frame
    def set_stream(self, stream_handle):
        """Run on this cudaStream_t.  None restores the context's own stream; the legacy
        default stream is cudaStreamLegacy (1), not 0."""
        if stream_handle == 0:
            raise AldicError("stream handle 0 means 'the context's own stream'; pass a created stream "
                             "(e.g. torch.cuda.Stream()) or cudaStreamLegacy (1)")
        self._check(self.lib.aldic_set_stream(self.h, C.c_void_p(stream_handle or 0)), "aldic_set_stream")

    def synchronize(self):
        self._check(self.lib.aldic_synchronize(self.h), "aldic_synchronize")

    @property
    def launches(self):
        return int(self.lib.aldic_launch_count(self.h))

    def set_iteration_cap(self, cap):
        """Iterations the one-warp solver pass spends on a subset before the multi-warp pass
        restarts it (default 8)."""
        self._check(self.lib.aldic_set_iteration_cap(self.h, int(cap)), "aldic_set_iteration_cap")

    def set_option(self, option, value):
        """A tuning option (aldic_set_option): OPT_ITERATION_CAP, OPT_STAGING, OPT_SLOW_WARPS,
        OPT_SEARCH_IMPL, OPT_SEARCH_CHUNK, OPT_AUTOTUNE."""
        self._check(self.lib.aldic_set_option(self.h, int(option), int(value)), "aldic_set_option")

    def get_option(self, option):
        v = C.c_int()
        self._check(self.lib.aldic_get_option(self.h, int(option), C.byref(v)), "aldic_get_option")
        return v.value

    def tuning_report(self):
        """The autotuner's choices (ALDIC_OPT_AUTOTUNE) as a dict."""
        import json

        buf = C.create_string_buffer(1 << 16)
        self._check(self.lib.aldic_tuning_report(self.h, buf, len(buf)), "aldic_tuning_report")
        return json.loads(buf.value.decode())

    def set_fp64_band(self, band, noise=_lib.DEFAULT_FP64_NOISE):
        """Margin around tol in which local_icgn re-decides a convergence test by an FP64
        re-solve of the subset: band x tol plus noise x the FP32 noise estimate of |b| (band 0
        disables; a huge band re-solves every subset)."""
        self._check(self.lib.aldic_set_fp64_band(self.h, float(band), float(noise)), "aldic_set_fp64_band")

    def set_profiling(self, on=True):
        """Record the device time of the correlation kernel of each integer_search call."""
        self._check(self.lib.aldic_set_profiling(self.h, 1 if on else 0), "aldic_set_profiling")

    def profile_read(self):
        """(total ms, number of recorded launches) since the last read; clears the record."""
        ms, n = C.c_double(), C.c_int()
        self._check(self.lib.aldic_profile_read(self.h, C.byref(ms), C.byref(n)), "aldic_profile_read")
        return ms.value, n.value

    def load_image_raw(self, slot, img, gridx, gridy, mask=None, want_stats=True, shape=None):
        k = _Keep()
        M, N = _img_shape(img, shape)
        gx = np.asarray(gridx, dtype=np.int32).ravel()
        gy = np.asarray(gridy, dtype=np.int32).ravel()
        ms = np.empty(2) if want_stats else None
        dtype_code = _np_dtype_code(img)
        npdt = {0: np.uint8, 1: np.uint16, 2: np.float32, 3: np.float64}[dtype_code]
        rc = self.lib.aldic_load_image_raw(self.h, slot, k.ptr(img, npdt, numel=M * N), dtype_code, M, N,
                                           C.c_void_p(gx.ctypes.data), C.c_void_p(gy.ctypes.data),
                                           k.ptr(mask, np.float64, numel=M * N),
                                           None if ms is None else C.c_void_p(ms.ctypes.data))
        self._check(rc, "aldic_load_image_raw")
        self.M, self.N = M, N
        return ms

    def load_image(self, slot, img):
        k = _Keep()
        M, N = img.shape
        self._check(self.lib.aldic_load_image(self.h, slot, k.ptr(img, np.float64), M, N), "aldic_load_image")
        self.M, self.N = M, N

    def set_mask(self, mask):
        k = _Keep()
        self._check(self.lib.aldic_set_mask(self.h, k.ptr(mask, np.float64), self.M, self.N), "aldic_set_mask")

    def compute_gradients(self):
        self._check(self.lib.aldic_compute_gradients(self.h), "aldic_compute_gradients")

    def set_gradients(self, dfdx, dfdy):
        k = _Keep()
        M6, N6 = dfdx.shape
        self._check(self.lib.aldic_set_gradients(self.h, k.ptr(dfdx, np.float64), k.ptr(dfdy, np.float64), M6, N6),
                    "aldic_set_gradients")

    def get_state(self, what):
        shape = (self.M, self.N) if what in (0, 1) else (self.M - 6, self.N - 6)
        out = np.empty(shape[0] * shape[1])
        self._check(self.lib.aldic_get_state(self.h, what, C.c_void_p(out.ctypes.data)), "aldic_get_state")
        return out.reshape(shape, order="F")

    # ------------------------------------------------------------ primitives
    def interp2(self, slot, X, Y):
        k = _Keep()
        X = np.asarray(X, dtype=np.float64)
        n = X.size
        Z, zp = k.out(n, np.float64)
        self._check(self.lib.aldic_interp2(self.h, slot, n, k.ptr(X, np.float64, "C"), k.ptr(Y, np.float64, "C"), zp),
                    "aldic_interp2")
        return Z.reshape(X.shape)

    def search_grid(self, gridx, gridy, winsize, step):
        gx = np.asarray(gridx, dtype=np.int32).ravel()
        gy = np.asarray(gridy, dtype=np.int32).ravel()
        nx, ny = C.c_int(), C.c_int()
        self._check(self.lib.aldic_search_grid(C.c_void_p(gx.ctypes.data), C.c_void_p(gy.ctypes.data), int(winsize),
                                               int(step), C.byref(nx), C.byref(ny)), "aldic_search_grid")
        return nx.value, ny.value

    def integer_search(self, search, gridx, gridy, winsize, step, out=None):
        """Whole-field search on the resident REF/DEF images.  Returns dict of nY x nX
        arrays (host), or fills `out`: a dict of CUDA tensors (asynchronously, on the
        context's stream) or of host numpy arrays (before the call returns)."""
        s = np.asarray(search, dtype=np.int32).ravel()
        if s.size == 1:
            s = np.array([s[0], s[0]], dtype=np.int32)
        gx = np.asarray(gridx, dtype=np.int32).ravel()
        gy = np.asarray(gridy, dtype=np.int32).ravel()
        nx, ny = self.search_grid(gx, gy, winsize, step)
        k = _Keep()
        if out is None:
            bufs = {name: k.out(nx * ny, np.float64) for name in ("x", "y", "u", "v", "phi")}
            ptrs = [bufs[nm][1] for nm in ("x", "y", "u", "v", "phi")]
        else:
            ptrs = [k.dst(out[nm], np.float64, nx * ny) for nm in ("x", "y", "u", "v", "phi")]
        rc = self.lib.aldic_integer_search(self.h, C.c_void_p(s.ctypes.data), C.c_void_p(gx.ctypes.data),
                                           C.c_void_p(gy.ctypes.data), int(winsize), int(step), *ptrs)
        self._check(rc, "aldic_integer_search")
        if out is not None:
            return out
        return {nm: bufs[nm][0].reshape((ny, nx), order="F") for nm in ("x", "y", "u", "v", "phi")}

    def local_icgn(self, variant, coords, U0, winsize, tol, want_H=True, want_mark=True, out=None, F0=None,
                   want_zncc=False):
        """LocalICGN / LocalICGNQuadtree loop body; F0 (4n) starts IC-GN from [F0 U0] (the
        learned initial guess) instead of the reference's [0 U0].  want_zncc (with F0) also
        returns each subset's ZNCC under its final warp, from IC-GN's last iteration (`zncc`; with `out`, into out["zncc"])."""
        k = _Keep()
        n = _count(coords, 2)
        if want_zncc and F0 is None:
            raise ValueError("want_zncc needs F0 (the learned-guess entry point)")
        zncc, zp = None, None
        if out is None:
            U, up = k.out(2 * n, np.float64)
            F, fp = k.out(4 * n, np.float64)
            H, hp = k.out(21 * n, np.float64) if want_H else (None, None)
            conv, cp = k.out(n, np.int32)
            mark, mp = k.out(n, np.uint8) if (want_mark and variant == _lib.QUADTREE) else (None, None)
            if want_zncc:
                zncc, zp = k.out(n, np.float64)
        else:
            up = k.dst(out["U"], np.float64, 2 * n)
            fp = k.dst(out["F"], np.float64, 4 * n)
            hp = k.dst(out.get("H"), np.float64, 21 * n)
            cp = k.dst(out["conv"], np.int32, n)
            mp = k.dst(out.get("mark"), np.uint8, n)
            if want_zncc:
                zp = k.dst(out["zncc"], np.float64, n)
        if F0 is None:
            rc = self.lib.aldic_local_icgn(self.h, int(variant), n, k.ptr(coords, np.float64, numel=2 * n),
                                           k.ptr(U0, np.float64, "C", numel=2 * n), int(winsize), float(tol), up, fp,
                                           hp, cp, mp)
        else:
            rc = self.lib.aldic_local_icgn_guess(self.h, int(variant), n, k.ptr(coords, np.float64, numel=2 * n),
                                                 k.ptr(U0, np.float64, "C", numel=2 * n),
                                                 k.ptr(F0, np.float64, "C", numel=4 * n), int(winsize), float(tol), up,
                                                 fp, hp, cp, mp, zp)
        self._check(rc, "aldic_local_icgn")
        if out is not None:
            return out
        return dict(U=U, F=F, H=None if H is None else H.reshape((n, 21), order="F"), conv=conv, markHole=mark,
                    zncc=zncc)

    def subset_zncc(self, coords, U, F, winsize, out=None):
        """ZNCC of each subset's window under the warp [F U] (NaN where it leaves the image)."""
        k = _Keep()
        n = _count(coords, 2)
        if out is None:
            z, zp = k.out(n, np.float64)
        else:
            z, zp = out, k.dst(out, np.float64, n)
        self._check(self.lib.aldic_subset_zncc(self.h, n, k.ptr(coords, np.float64, numel=2 * n),
                                               k.ptr(U, np.float64, "C", numel=2 * n),
                                               k.ptr(F, np.float64, "C", numel=4 * n), int(winsize), zp),
                    "aldic_subset_zncc")
        return z

    def fallback_select(self, conv, zncc, zncc_min, out, count=None):
        """Indices (0-based, in no fixed order) of the subsets with conv outside 1..100 or
        zncc below zncc_min (or NaN) into `out` (int32, n entries of room: a CUDA tensor or a
        writeable numpy array); returns their number (waits for the device).  With `count` (a
        1-entry int64 CUDA tensor) the number goes there instead, queued on the context's
        stream without a wait, and the call returns None."""
        k = _Keep()
        n = int(conv.numel() if _is_torch(conv) else np.asarray(conv).size)
        if count is not None:
            if not (_is_torch(count) and count.is_cuda):
                raise ValueError("count must be a 1-entry int64 CUDA tensor")
            self._check(self.lib.aldic_fallback_select(self.h, n, k.ptr(conv, np.int32), k.ptr(zncc, np.float64),
                                                       float(zncc_min), k.dst(out, np.int32, n),
                                                       k.ptr(count, np.int64, numel=1)), "aldic_fallback_select")
            return None
        cnt = C.c_int64()
        self._check(self.lib.aldic_fallback_select(self.h, n, k.ptr(conv, np.int32), k.ptr(zncc, np.float64),
                                                   float(zncc_min), k.dst(out, np.int32, n), C.byref(cnt)),
                    "aldic_fallback_select")
        return int(cnt.value)

    def integer_search_list(self, search, gridx, gridy, winsize, step, grid_idx, out=None):
        """The integer search on the grid subsets grid_idx (i + j nX) only: dict of n-entry
        arrays x, y, u, v, phi in list order (or the CUDA tensors of `out`)."""
        k = _Keep()
        s = np.asarray(search, dtype=np.int32).ravel()
        if s.size == 1:
            s = np.array([s[0], s[0]], dtype=np.int32)
        n = int(grid_idx.numel() if _is_torch(grid_idx) else np.asarray(grid_idx).size)
        names = ("x", "y", "u", "v", "phi")
        if out is None:
            bufs = [k.out(n, np.float64) for _ in names]
            res, ptrs = {nm: b[0] for nm, b in zip(names, bufs)}, [b[1] for b in bufs]
        else:
            res, ptrs = out, [k.dst(out[nm], np.float64, n) for nm in names]
        rc = self.lib.aldic_integer_search_list(self.h, k.ptr(s, np.int32), k.ptr(np.asarray(gridx), np.int32),
                                                k.ptr(np.asarray(gridy), np.int32), int(winsize), int(step), n,
                                                k.ptr(grid_idx, np.int32), *ptrs)
        self._check(rc, "aldic_integer_search_list")
        return res

    def net_extract(self, coords, X):
        """The proposal network's inputs of the subsets at coords into X, a CUDA bf16 tensor
        (n, 64, 64, 2)."""
        k = _Keep()
        n = _count(coords, 2)
        self._check(self.lib.aldic_net_extract(self.h, n, k.ptr(coords, np.float64, numel=2 * n),
                                               C.c_void_p(X.data_ptr())), "aldic_net_extract")
        return X

    def subpb1(self, variant, coords, UOld, FOld, vdual, mu, tol, winsize=0, winsize_list=None, HPar=None, out=None):
        """Subpb1 / Subpb1Quadtree local step.  With `out` (dict of CUDA tensors U (2n), conv (n))
        and device inputs the call stays on the device and returns `out` asynchronously."""
        k = _Keep()
        n = _count(coords, 2)
        if out is None:
            U, up = k.out(2 * n, np.float64)
            conv, cp = k.out(n, np.int32)
        else:
            up = k.dst(out["U"], np.float64, 2 * n)
            cp = k.dst(out["conv"], np.int32, n)
        wl = None if winsize_list is None else k.ptr(winsize_list, np.int32, numel=2 * n)  # n x 2 (wx, wy)
        rc = self.lib.aldic_subpb1(self.h, int(variant), n, k.ptr(coords, np.float64, numel=2 * n),
                                   k.ptr(UOld, np.float64, "C", numel=2 * n), k.ptr(FOld, np.float64, "C", numel=4 * n),
                                   k.ptr(vdual, np.float64, "C", numel=2 * n), wl, int(winsize),
                                   k.ptr(HPar, np.float64), float(mu), float(tol), up, cp)
        self._check(rc, "aldic_subpb1")
        if out is not None:
            return out
        return dict(U=U, conv=conv)

    def epipolar_icgn(self, pts, winsize, tol):
        k = _Keep()
        n = _count(pts, 2)
        z, zp = k.out(n, np.float64)
        self._check(self.lib.aldic_epipolar_icgn(self.h, n, k.ptr(pts, np.float64), int(winsize), float(tol), zp),
                    "aldic_epipolar_icgn")
        return z

    def inpaint_nans(self, A, info=False):
        """inpaint_nans(A, 4) (spring analogy).  A host array is returned as a new filled
        array; a CUDA tensor (with shape=(m, n) implied by a 2-D tensor, column-major data)
        is filled in place.  info=True also returns (NaN entries, CG iterations, converged)."""
        k = _Keep()
        nfo = (C.c_int32 * 3)()
        if _is_torch(A):
            if A.dim() != 2:
                raise AldicError("device grids must be 2-D tensors (n, m) holding the column-major m x n grid")
            n, m = A.shape  # row-major (n, m) == column-major m x n
            rc = self.lib.aldic_inpaint_nans(self.h, int(m), int(n), k.ptr(A, np.float64), nfo if info else None)
            self._check(rc, "aldic_inpaint_nans")
            return (A, tuple(nfo)) if info else A
        a = np.array(A, dtype=np.float64, order="F", copy=True)
        m, n = a.shape
        rc = self.lib.aldic_inpaint_nans(self.h, int(m), int(n), C.c_void_p(a.ctypes.data), nfo if info else None)
        self._check(rc, "aldic_inpaint_nans")
        return (a, tuple(nfo)) if info else a

    def remove_outliers(self, u, v, thr=100.0, maxit=0, info=False):
        """funRemoveOutliers(u, v, cc, 0, thr): the median test and inpaint of the search grids.
        Host arrays (m x n) are returned as new arrays (u, v); CUDA tensors (2-D, (n, m)
        holding the column-major m x n grids) are updated in place.  info=True also returns
        (removed, NaN holes, method-3 iterations, converged)."""
        k = _Keep()
        nfo = (C.c_int32 * 4)()
        if _is_torch(u):
            if u.dim() != 2 or tuple(v.shape) != tuple(u.shape):
                raise AldicError("device grids must be two 2-D tensors (n, m) holding column-major m x n grids")
            n, m = u.shape
            rc = self.lib.aldic_remove_outliers(self.h, int(m), int(n), k.ptr(u, np.float64), k.ptr(v, np.float64),
                                                float(thr), int(maxit), nfo if info else None)
            self._check(rc, "aldic_remove_outliers")
            return (u, v, tuple(nfo)) if info else (u, v)
        a = np.array(u, dtype=np.float64, order="F", copy=True)
        b = np.array(v, dtype=np.float64, order="F", copy=True)
        if a.ndim != 2 or a.shape != b.shape:
            raise AldicError("u and v must be 2-D grids of one shape")
        m, n = a.shape
        rc = self.lib.aldic_remove_outliers(self.h, int(m), int(n), C.c_void_p(a.ctypes.data),
                                            C.c_void_p(b.ctypes.data), float(thr), int(maxit), nfo if info else None)
        self._check(rc, "aldic_remove_outliers")
        return (a, b, tuple(nfo)) if info else (a, b)

    @staticmethod
    def _elements(elements):
        if _is_torch(elements):
            return elements, _count(elements, 8)  # an (8, n_el) int32 tensor: the column-major n_el x 8 table
        E = np.asarray(elements)
        if E.ndim != 2 or E.shape[1] != 8:
            raise AldicError("elements must be an n_el x 8 array (corners 1-4, mid-side nodes 5-8, 0 = none)")
        return E, int(E.shape[0])

    def subpb2_set_mesh(self, n, elements, dirichlet=None):
        """Keep a global-step mesh (n nodes; elements n_el x 8; dirichlet node numbers)
        resident for subpb2(..., elements=None, ...)."""
        k = _Keep()
        E, n_el = self._elements(elements)
        d = np.zeros(0, np.int32) if dirichlet is None or np.size(dirichlet) == 0 else \
            np.ravel(np.asarray(dirichlet)).astype(np.int32)
        rc = self.lib.aldic_subpb2_set_mesh(self.h, int(n), n_el, k.ptr(E, np.int32), int(d.size),
                                            k.ptr(d, np.int32) if d.size else None)
        self._check(rc, "aldic_subpb2_set_mesh")
        self._sp2_nel = n_el

    def subpb2(self, coords, elements, gauss_order, beta, mu, U, F, alpha=0.0, dirichlet=None, tol=0.0, maxit=0,
               out=None, info=False):
        """Subpb2Quadtree's global finite-element step: coords (n x 2), elements (n_el x 8,
        1-based, 0 = no mid-side node), U (2n), F (4n), dirichlet node numbers (1-based).
        Returns Uhat (2n), or fills `out`; info=True also returns (iterations, converged)."""
        k = _Keep()
        n = _count(coords, 2)
        if elements is None:  # the resident mesh of subpb2_set_mesh
            E, n_el = None, self._sp2_nel
            if dirichlet is not None:
                raise AldicError("the resident mesh carries its dirichlet nodes")
        else:
            E, n_el = self._elements(elements)
        if dirichlet is None:
            d = np.zeros(0, np.int32)
        elif _is_torch(dirichlet):
            d = dirichlet.reshape(-1)
        else:
            d = np.ravel(np.asarray(dirichlet)).astype(np.int32)
        nd = int(d.numel() if _is_torch(d) else d.size)
        if out is None:
            Uh, op = k.out(2 * n, np.float64)
        else:
            Uh, op = out, k.dst(out, np.float64, 2 * n)
        nfo = (C.c_int32 * 2)()
        rc = self.lib.aldic_subpb2(self.h, n, k.ptr(coords, np.float64), n_el,
                                   None if E is None else k.ptr(E, np.int32), int(gauss_order),
                                   float(beta), float(mu), float(alpha), k.ptr(U, np.float64, numel=2 * n),
                                   k.ptr(F, np.float64, numel=4 * n), nd, k.ptr(d, np.int32) if nd else None,
                                   float(tol), int(maxit), op, nfo)
        self._check(rc, "aldic_subpb2")
        return (Uh, tuple(nfo)) if info else Uh

    def init_u0(self, u, v, out=None, index=0):
        """Init(u, v, Phi, x, y, index): inpaint the search grids (ny x nx, left unchanged;
        index 1 adds the spring outlier passes) and return U0 (2 nx ny, mesh order), or fill
        `out` (a CUDA tensor or host array)."""
        k = _Keep()
        if _is_torch(u):
            if u.dim() != 2:
                raise AldicError("device grids must be 2-D tensors (nx, ny) holding the column-major ny x nx grid")
            nx, ny = u.shape
        else:
            ny, nx = np.shape(u)
        if out is None:
            U0, op = k.out(2 * nx * ny, np.float64)
        else:
            U0, op = out, k.dst(out, np.float64, 2 * nx * ny)
        rc = self.lib.aldic_init_u0(self.h, int(ny), int(nx), k.ptr(u, np.float64, numel=nx * ny),
                                    k.ptr(v, np.float64, numel=nx * ny), int(index), op)
        self._check(rc, "aldic_init_u0")
        return U0

    def undistort_points(self, pts, K, radial, tangential=None):
        """MATLAB undistortPoints for one camera: pts (n x 2, 1-based pixels) through the
        inverse of the radial (2 or 3 coefficients) and tangential (p1, p2) lens model of K."""
        k = _Keep()
        p = np.asarray(pts, dtype=np.float64).reshape(-1, 2)
        n = p.shape[0]
        rad = np.asarray(radial, dtype=np.float64).ravel()
        out, op = k.out(2 * n, np.float64)
        tan = None if tangential is None else k.ptr(np.ravel(tangential), np.float64)
        rc = self.lib.aldic_undistort_points(self.h, n, k.ptr(p, np.float64), k.ptr(np.asarray(K, np.float64), np.float64),
                                             k.ptr(rad, np.float64), int(rad.size), tan, op)
        self._check(rc, "aldic_undistort_points")
        return out.reshape((n, 2), order="F")

    def triangulate(self, pairs, KL, KR, R, T, out=None):
        k = _Keep()
        n = _count(pairs, 4)
        if out is None:
            xyz, xp = k.out(3 * n, np.float64)
            err, ep = k.out(n, np.float64)
        else:
            xp = k.dst(out["xyz"], np.float64, 3 * n)
            ep = k.dst(out.get("err"), np.float64, n)
        rc = self.lib.aldic_triangulate(self.h, n, k.ptr(pairs, np.float64, numel=4 * n), k.ptr(KL, np.float64),
                                        k.ptr(KR, np.float64), k.ptr(R, np.float64), k.ptr(np.ravel(T), np.float64),
                                        xp, ep)
        self._check(rc, "aldic_triangulate")
        if out is not None:
            return out
        return xyz.reshape((n, 3), order="F"), err


_CTX = {}


def default_context(device: int = 0) -> Context:
    if device not in _CTX:
        _CTX[device] = Context(device)
    return _CTX[device]


# ==================================================================================
# MATLAB-signature mirrors
# ==================================================================================
def funNormalizeImg(Img, gridxyROIRange, ctx: Context | None = None):
    """[ImgNormalized, gridxyROIRange] = funNormalizeImg(Img, gridxyROIRange)
    (func/funNormalizeImg.m:1-127).  Img: list of raw images."""
    ctx = ctx or default_context()
    gx = list(gridxyROIRange["gridx"])
    gy = list(gridxyROIRange["gridy"])
    M, N = Img[0].shape
    gx = [max(gx[0], 1), min(gx[1], M)]
    gy = [max(gy[0], 1), min(gy[1], N)]
    out = []
    for im in Img:
        ctx.load_image_raw(_lib.SLOT_DEF, im, gx, gy)
        out.append(ctx.get_state(1))
    return out, {"gridx": gx, "gridy": gy}


def funImgGradient(ImgRef, ImgDef=None, ImgRefMask=None, ctx: Context | None = None):
    """Df = funImgGradient(ImgRef, ImgDef, ImgRefMask) (func/funImgGradient.m:50-83)."""
    ctx = ctx or default_context()
    ImgRef = np.asarray(ImgRef, dtype=np.float64)
    M, N = ImgRef.shape
    ctx.load_image(_lib.SLOT_REF, ImgRef)
    mask = np.ones((M, N)) if ImgRefMask is None else np.asarray(ImgRefMask, dtype=np.float64)
    ctx.set_mask(mask)
    ctx.compute_gradients()
    return {"DfDx": ctx.get_state(2), "DfDy": ctx.get_state(3), "ImgRefMask": mask, "DfCropWidth": 3,
            "imgSize": (M, N), "DfAxis": [4, M - 3, 4, N - 3]}


def ba_interp2_spline(F, X, Y, method="cubicspline", ctx: Context | None = None):
    """Z = ba_interp2_spline(F, X, Y) (ba_interp2_spline.cpp:418-435); X = dim-2 and
    Y = dim-1 coordinates (1-based)."""
    ctx = ctx or default_context()
    ctx.load_image(_lib.SLOT_DEF, np.asarray(F, dtype=np.float64))
    return ctx.interp2(_lib.SLOT_DEF, X, Y)


def Init(u, v, Phi=None, x=None, y=None, index=0, ctx: Context | None = None):
    """Init(u, v, Phi, x, y, index) (func/Init.m): inpaint_nans(., 4) of u and v, with
    index 1 the three spring outlier passes, and U0 in mesh order.  The stereo and temporal
    drivers call index 0."""
    ctx = ctx or default_context()
    return ctx.init_u0(u, v, index=index)


def funIntegerSearch(f, g, tempSizeOfSearchRegion, gridx, gridy, winsize, winstepsize, tempNoOfInitPt=0,
                     ctx: Context | None = None):
    """[x, y, u, v, cc] = funIntegerSearch(f, g, search, gridx, gridy, winsize, step, 0)
    (func/funIntegerSearch.m:2-98).  Only the whole-field mode (0) is on the device."""
    if tempNoOfInitPt != 0:
        raise AldicError("funIntegerSearch: only the whole-field mode (tempNoOfInitPt = 0) is implemented")
    ctx = ctx or default_context()
    ctx.load_image(_lib.SLOT_REF, np.asarray(f, dtype=np.float64))
    ctx.load_image(_lib.SLOT_DEF, np.asarray(g, dtype=np.float64))
    w = int(np.ravel(winsize)[0])
    st = int(np.ravel(winstepsize)[0])
    r = ctx.integer_search(tempSizeOfSearchRegion, gridx, gridy, w, st)
    return r["x"], r["y"], r["u"], r["v"], {"max": r["phi"], "A": []}


def Subpb2Quadtree(DICmesh, GaussPtOrder, beta, mu, U, F, udual=None, vdual=None, alpha=0.0, winstepsize=None,
                   waitBarDisplayOrNot=0, ctx: Context | None = None):
    """[Uhat] = Subpb2Quadtree(DICmesh, GaussPtOrder, beta, mu, U, F, udual, vdual, alpha,
    winstepsize, waitBarDisplayOrNot) (func_quadtree/Subpb2Quadtree.m): ALDIC's global
    finite-element step on the device.  DICmesh holds coordinatesFEM (n x 2),
    elementsFEM (n_el x 8) and dirichlet (node numbers, may be empty); a non-empty neumann
    list raises (the drivers' quadtree meshes carry none).  udual, vdual and winstepsize do
    not enter the result (the reference multiplies the duals by 0; winstepsize scales only
    the neumann term)."""
    neu = DICmesh.get("neumann")
    if neu is not None and np.size(neu) > 0:
        raise AldicError("Subpb2Quadtree: neumann boundary terms are not implemented")
    ctx = ctx or default_context()
    dirichlet = DICmesh.get("dirichlet")
    return ctx.subpb2(DICmesh["coordinatesFEM"], DICmesh["elementsFEM"], GaussPtOrder, beta, mu, U, F, alpha=alpha,
                      dirichlet=None if dirichlet is None or np.size(dirichlet) == 0 else dirichlet)


def subpb2_beta(betaList, errs):
    """The reference's beta for the first frame (func/TemporalMatch_quadtree_ST1.m:274-294):
    |U1 - U2| over the three-entry beta list normalised by its mean and standard deviation,
    the minimum's beta, or, with the minimum in the middle, the vertex of the parabola in
    log10(beta) through the three points (MATLAB's fit(..., 'poly2') there, whose try falls
    to the list's beta at an end)."""
    e = np.asarray(errs, dtype=np.float64)
    sd = e.std(ddof=1)
    if not (np.isfinite(sd) and sd > 0):  # MATLAB's min over NaN picks the first entry
        return betaList[0]
    z = (e - e.mean()) / sd
    k = int(np.argmin(z))
    if k != 1:
        return betaList[k]
    p = np.polyfit(np.log10(betaList), z, 2)
    return 10 ** (-p[1] / 2 / p[0])


def ALDICFrameQuadtree(fNormalized, gNormalized, fNormalizedMask, DICpara, ImgSeqNum=2, file_name=None,
                       shapeFuncOrder=1, ctx: Context | None = None, seed=None):
    """One frame of func/TemporalMatch_quadtree_ST1.m (:41-390, sections 3 to 6) in its
    default form (accumulative, whole-field search initial guess, UseGlobal): gradients of
    the reference frame; IntegerSearchQuadtree (search and bad-point removal), MeshSetUp, Init
    and the nodes outside the mask set NaN (:108-160); GenerateQuadtreeMesh with
    elementMinSize = DICpara['winsizeMin'] (:163-169); LocalICGNQuadtree with tol 1e-2 and
    its fills, then the section-4 fills of U and F ('natural', 'none', :200-240); the global
    step with mu = 1e-3, alpha = 0, Gauss order 2, beta tuned over [1e-3 1e-2 1e-1]
    mean(winstepsize)^2 mu at frame 2 (DICpara['beta'] or the list's first entry later,
    :266-306), the hole-strain nodes held at the local result, the duals (:313-323); two ADMM
    rounds of Subpb1Quadtree + Subpb2Quadtree (:333-389).  seed = (coords, U n x 2) replaces
    the search by the natural-neighbour interpolation of an earlier result onto the search
    grid ('natural', 'none', NaN -> 0, cc.max = 1; the 'reuseLast' initial guess, :112-128).
    Returns a dict: DICmesh, DICmesh_nonQuadtree, U (USubpb2), USubpb1, FSubpb1, beta,
    markCoordHoleStrain, DICpara.  DICpara['Smooth2DTimes'] (default 0) smooths USubpb1
    before the global step and USubpb2 in each ADMM round that many times, and
    DICpara['DispSmoothness'] > 1e-6 smooths the first global result once
    (funSmoothDispQuadtree, :257-263, :310, :355-357)."""
    ctx = ctx or default_context()
    n_smooth = int(DICpara.get("Smooth2DTimes", 0) or 0)
    disp_smooth = float(DICpara.get("DispSmoothness", 0) or 0) > 1e-6
    fN = np.asarray(fNormalized, dtype=np.float64)
    gN = np.asarray(gNormalized, dtype=np.float64)
    fMask = np.asarray(fNormalizedMask, dtype=np.float64)
    Df = funImgGradient(fN, fN, fMask, ctx=ctx)
    if seed is None:
        DICpara, x0, y0, u, v, cc = IntegerSearchQuadtree(fN, gN, file_name, DICpara, ImgSeqNum, ctx=ctx)
    else:  # the grid of funIntegerSearch (XList / YList, :114-118) from the earlier result
        w = int(np.ravel(DICpara["winsize"])[0])
        st = int(np.ravel(DICpara["winstepsize"])[0])
        roi = DICpara["gridxyROIRange"]
        xl = np.arange(roi["gridx"][0], roi["gridx"][1] - w - st + 1, st, dtype=np.float64)
        yl = np.arange(roi["gridy"][0], roi["gridy"][1] - w - st + 1, st, dtype=np.float64)
        X, Y = np.meshgrid(xl, yl, indexing="ij")
        pc, pu = np.asarray(seed[0], dtype=np.float64), np.asarray(seed[1], dtype=np.float64).reshape(-1, 2)
        ok = ~np.isnan(pu[:, 0])
        nn = _fill.NaturalNeighbor(pc[ok], "none")
        uv = nn(np.stack([X.ravel(), Y.ravel()], 1), pu[ok])
        uv[np.isnan(uv)] = 0.0
        x0, y0 = X.T, Y.T  # nY x nX, as funIntegerSearch returns them
        u, v = uv[:, 0].reshape(X.shape).T, uv[:, 1].reshape(X.shape).T
        cc = {"max": np.ones(u.shape)}
    mesh0 = MeshSetUp(x0, y0, DICpara)
    U0 = np.array(Init(u, v, cc["max"], mesh0["x0"], mesh0["y0"], 0, ctx=ctx), dtype=np.float64)
    C0 = mesh0["coordinatesFEM"]
    off = np.flatnonzero(fMask[np.floor(C0[:, 0] + 0.5).astype(np.int64) - 1,
                               np.floor(C0[:, 1] + 0.5).astype(np.int64) - 1] < 1)
    U0[2 * off] = np.nan
    U0[2 * off + 1] = np.nan
    mesh0["elementMinSize"] = DICpara["winsizeMin"]
    mesh, DICpara, U0 = GenerateQuadtreeMesh(U0, Df, fMask, mesh0, DICpara)
    C = mesh["coordinatesFEM"]
    # section 4: the local step and its fills
    U1, F1, _, _, _, _, hole = LocalICGNQuadtree(U0, C, Df, fN, gN, DICpara, "GaussNewton", 1e-2, shapeFuncOrder,
                                                 ctx=ctx)
    U1 = U1.reshape(-1, 2)
    if np.isnan(U1[:, 0]).any() and (~np.isnan(U1[:, 0])).sum() > 10:
        U1 = _fill.fill_nans_natural(C, U1, "none")
    F1 = F1.reshape(-1, 4)
    if np.isnan(F1[:, 0]).any() and (~np.isnan(F1[:, 0])).sum() > 10:
        F1 = _fill.fill_nans_natural(C, F1, "none")
    U1, F1 = U1.ravel(), F1.ravel()
    for _ in range(n_smooth):
        U1 = _smooth.funSmoothDispQuadtree(U1, mesh, DICpara)
    # section 5: the global step
    mu, alpha, order = 1e-3, 0.0, 2
    step = float(np.mean(np.ravel(DICpara["winstepsize"])))
    betaList = [c * step ** 2 * mu for c in (1e-3, 1e-2, 1e-1)]
    hdof = np.concatenate([2 * np.asarray(hole, dtype=np.int64), 2 * np.asarray(hole, dtype=np.int64) + 1])
    U2 = None
    if ImgSeqNum == 2:
        errs = []
        for bt in betaList:
            U2 = Subpb2Quadtree(mesh, order, bt, mu, U1, F1, None, None, alpha, step, 0, ctx=ctx)
            errs.append(np.linalg.norm(U1 - U2))
        beta = subpb2_beta(betaList, errs)
    else:
        beta = DICpara.get("beta", 1e-3 * step ** 2 * mu)
    if U2 is None or abs(beta - betaList[-1]) > np.finfo(float).eps:
        U2 = Subpb2Quadtree(mesh, order, beta, mu, U1, F1, None, None, alpha, step, 0, ctx=ctx)
    U2 = np.array(U2)
    if disp_smooth:
        U2 = _smooth.funSmoothDispQuadtree(U2, mesh, DICpara)
    U2[hdof] = U1[hdof]
    F2 = F1
    vdual = U2 - U1
    # section 6: two ADMM rounds
    para = dict(DICpara, winsize_List=np.full((C.shape[0], 2), int(np.ravel(DICpara["winsize"])[0]), np.int32))
    for ALSolveStep in (2, 3):
        U1, _, _, _, _ = Subpb1Quadtree(U2, F2, np.zeros(4 * C.shape[0]), vdual, C, Df, fN, gN, mu, beta, None,
                                        ALSolveStep, para, "GaussNewton", 1e-2, ctx=ctx)
        U2 = np.array(Subpb2Quadtree(mesh, order, beta, mu, U1, F1, None, None, alpha, step, 0, ctx=ctx))
        for _ in range(n_smooth):
            U2 = _smooth.funSmoothDispQuadtree(U2, mesh, DICpara)
        U2[hdof] = U1[hdof]
        vdual = U2 - U1
    return {"DICmesh": mesh, "DICmesh_nonQuadtree": mesh0, "U": U2, "USubpb1": U1, "FSubpb1": F1, "beta": beta,
            "markCoordHoleStrain": hole, "DICpara": DICpara}


def TemporalMatch_quadtree_ST1(DICpara, file_name, ImgMask, ImgNormalized, RD=None, StereoInfo=None,
                               camera0OrNot="camera0", shapeFuncOrder=1, ctx: Context | None = None):
    """[RD] = TemporalMatch_quadtree_ST1(DICpara, file_name, ImgMask, ImgNormalized, RD,
    StereoInfo, camera0OrNot, shapeFuncOrder) (func/TemporalMatch_quadtree_ST1.m) with the
    global step, frame by frame through ALDICFrameQuadtree.
    * Accumulative mode (DICIncOrNot 0): frame k >= 2 against frame 1 (masked by ImgMask[0],
      the deformed frame unmasked, :48-53); ResultDisp_acc holds USubpb2; ResultDisp the field
      at the first frame's mesh ('camera0') or carried to RD['Coordinates_corr'] by
      natural-neighbour interpolation ('notCamera0', 'natural', 'none', :401-426);
      DICpara['TemporalInitGuess'] = 'reuseLast' seeds frames 3+ from the previous result when
      more than half of it is valid (:62-81).
    * Incremental mode (DICIncOrNot 1): frame k against frame k - 1, both masked by their own
      masks (:43-47), a mesh per frame; ResultDisp_inc holds USubpb2, and ResultDisp
      accumulates it at the tracked points (the first frame's mesh, or the matched points,
      moved by the displacement so far; 'natural', 'none', :434-479).
    For 'notCamera0' the search ROI is the reference frame mask's bounding box
    (localizeDICparaForFrame, :513-531).  RD gains ResultFEMesh, ResultFEMeshEachFrame,
    ResultDisp and ResultDisp_acc / ResultDisp_inc (and ResultDisp_corr for 'notCamera0' in
    the accumulative mode)."""
    inc = int(DICpara.get("DICIncOrNot", 0))
    if inc not in (0, 1):
        raise AldicError("DICIncOrNot must be 0 (accumulative) or 1 (incremental)")
    if camera0OrNot not in ("camera0", "notCamera0"):
        raise AldicError("camera0OrNot must be 'camera0' or 'notCamera0'")
    RD = dict(RD or {})
    for key in ("ResultDisp_acc", "ResultDisp_inc", "ResultDisp", "ResultDisp_corr", "ResultFEMesh",
                "ResultFEMeshEachFrame"):
        RD[key] = list(RD.get(key, []))

    def localize(para, mask):
        para = dict(para, ImgRefMask=mask)
        if camera0OrNot == "notCamera0":
            rows, cols = np.nonzero(mask)
            para["gridxyROIRange"] = {"gridx": [int(rows.min()) + 1, int(rows.max()) + 1],
                                      "gridy": [int(cols.min()) + 1, int(cols.max()) + 1]}
        return para

    def carry(src, Uq, pts):
        ok = ~np.isnan(Uq[:, 0])
        return _fill.NaturalNeighbor(src[ok], "none")(np.asarray(pts, dtype=np.float64), Uq[ok])

    para = dict(DICpara)
    for k in range(2, len(ImgNormalized) + 1):
        if inc:
            fMask = np.asarray(ImgMask[k - 2], dtype=np.float64)
            gMask = np.asarray(ImgMask[k - 1], dtype=np.float64)
            fN = np.asarray(ImgNormalized[k - 2], dtype=np.float64) * fMask
            gN = np.asarray(ImgNormalized[k - 1], dtype=np.float64) * gMask
        else:
            fMask = np.asarray(ImgMask[0], dtype=np.float64)
            fN = np.asarray(ImgNormalized[0], dtype=np.float64) * fMask
            gN = np.asarray(ImgNormalized[k - 1], dtype=np.float64)
        para = localize(para, fMask)
        seed = None
        if not inc and para.get("TemporalInitGuess") == "reuseLast" and k >= 3:
            prev = np.asarray(RD["ResultDisp"][k - 3]["U"], dtype=np.float64).reshape(-1, 2)
            pc = np.asarray(RD["ResultFEMeshEachFrame"][0]["coordinatesFEM"], dtype=np.float64)
            if prev.shape[0] == pc.shape[0] and 1 - np.isnan(prev[:, 0]).mean() > 0.5:
                seed = (pc, prev)
        r = ALDICFrameQuadtree(fN, gN, fMask, para, k, file_name, shapeFuncOrder, ctx=ctx, seed=seed)
        para = dict(r["DICpara"], gridxyROIRange=para["gridxyROIRange"])
        if k == 2 or inc:
            m0, mq = r["DICmesh_nonQuadtree"], r["DICmesh"]
            RD["ResultFEMesh"].append({"coordinatesFEM": m0["coordinatesFEM"], "elementsFEM": m0["elementsFEM"],
                                       "winsize": para["winsize"], "winstepsize": para["winstepsize"],
                                       "gridxyROIRange": para["gridxyROIRange"]})
            RD["ResultFEMeshEachFrame"].append({"coordinatesFEM": mq["coordinatesFEM"],
                                                "elementsFEM": mq["elementsFEM"]})
        U = np.asarray(r["U"], dtype=np.float64)
        Uq = U.reshape(-1, 2)
        first = np.asarray(RD["ResultFEMeshEachFrame"][0]["coordinatesFEM"], dtype=np.float64)
        if not inc:
            RD["ResultDisp_acc"].append({"U": U})
            if camera0OrNot == "camera0":
                RD["ResultDisp"].append({"U": Uq})
            else:
                RD["ResultDisp"].append({"U": carry(first, Uq, RD["Coordinates_corr"])})
                RD["ResultDisp_corr"].append({"U": Uq})
            continue
        RD["ResultDisp_inc"].append({"U": U})
        src = np.asarray(RD["ResultFEMeshEachFrame"][k - 2]["coordinatesFEM"], dtype=np.float64)
        base = first if camera0OrNot == "camera0" else np.asarray(RD["Coordinates_corr"], dtype=np.float64)
        if k == 2:
            RD["ResultDisp"].append({"U": Uq if camera0OrNot == "camera0" else carry(src, Uq, base)})
        else:
            prev = np.asarray(RD["ResultDisp"][k - 3]["U"], dtype=np.float64)
            RD["ResultDisp"].append({"U": prev + carry(src, Uq, base + prev)})
    return RD


def funRemoveOutliers(u, v, cc, qDICOrNot, Thr0, ctx: Context | None = None):
    """[u, v, cc] = funRemoveOutliers(u, v, cc, qDICOrNot, Thr0) (func/funRemoveOutliers.m) for
    the form the drivers use, qDICOrNot = 0 and Thr0 > 0 (func_quadtree/IntegerSearchQuadtree.m:
    158-160): the median test (:44-64) and inpaint (:66-72) on the device.  The q-factor branch
    (qDICOrNot = 1) and the prompting branches (Thr0 = 0, |qDICOrNot| > 0) raise."""
    if qDICOrNot != 0:
        raise AldicError("funRemoveOutliers: only qDICOrNot = 0 is implemented (the q-factor branch prompts)")
    if Thr0 is None or np.size(Thr0) == 0 or float(np.ravel(Thr0)[0]) == 0.0:
        raise AldicError("funRemoveOutliers: Thr0 = 0 prompts for a threshold in the reference; pass one")
    ctx = ctx or default_context()
    u2, v2 = ctx.remove_outliers(u, v, float(np.ravel(Thr0)[0]))
    return u2, v2, cc


def IntegerSearchQuadtree(ImgRef, ImgDef, file_name, DICpara, ImgSeqNum, ctx: Context | None = None):
    """[DICpara, x0, y0, u, v, cc] = IntegerSearchQuadtree(ImgRef, ImgDef, file_name, DICpara,
    ImgSeqNum) (func_quadtree/IntegerSearchQuadtree.m), whole-field mode
    (InitFFTSearchMethod 1) or all-zero initial guesses (3).  The search distance follows :48-62 -- stereo (ImgSeqNum -1):
    StereoSearchDistance, else NewFFTSearchDistance; temporal (ImgSeqNum >= 2):
    TemporalSearchDistance, else NewFFTSearchDistance -- and a missing one raises instead of
    prompting.  The whole-field search runs on the device (:93); grid points whose rounded
    position is outside DICpara['ImgRefMask'] become NaN (:100-111), then the median-test
    bad-point removal funRemoveOutliers(u, v, cc, 0, 100) runs on the device (:158-160; the
    NaN holes stay NaN for Init to fill)."""
    method = DICpara.get("InitFFTSearchMethod", 1)
    if method == 3:  # all initial guesses zero (:213-222): the ROI grid at winstepsize, no search
        roi = DICpara["gridxyROIRange"]
        st = int(np.ravel(DICpara["winstepsize"])[0])
        xs = np.arange(roi["gridx"][0], roi["gridx"][1] + 1, st, dtype=np.float64)
        ys = np.arange(roi["gridy"][0], roi["gridy"][1] + 1, st, dtype=np.float64)
        x0 = np.tile(xs, (ys.size, 1))
        y0 = np.tile(ys[:, None], (1, xs.size))
        z = np.zeros(x0.shape)
        return (dict(DICpara, InitFFTSearchMethod=3, SizeOfFFTSearchRegion=np.array([0, 0])), x0, y0, z, z.copy(),
                {"max": np.ones(x0.shape)})
    if method != 1:
        raise AldicError("IntegerSearchQuadtree: the whole-field (1) and zero (3) initial guesses are implemented; "
                         "modes 0 and 2 need interactive input in the reference")
    keys = ("StereoSearchDistance", "NewFFTSearchDistance") if ImgSeqNum == -1 else \
        ("TemporalSearchDistance", "NewFFTSearchDistance") if ImgSeqNum >= 2 else ()
    s = None
    for key in keys:
        if DICpara.get(key) is not None and np.size(DICpara[key]) > 0:
            s = DICpara[key]
            break
    if s is None:
        raise AldicError("IntegerSearchQuadtree: no search distance in DICpara for this image (the reference prompts)")
    s = np.ravel(np.asarray(s, dtype=np.int64))
    s = np.array([s[0], s[0]]) if s.size == 1 else s[:2]
    roi = DICpara["gridxyROIRange"]
    x0, y0, u, v, cc = funIntegerSearch(ImgRef, ImgDef, s, roi["gridx"], roi["gridy"], DICpara["winsize"],
                                        DICpara["winstepsize"], 0, ctx=ctx)
    mask = DICpara.get("ImgRefMask")
    if mask is not None:
        mask = np.asarray(mask)
        # MATLAB round (half away from zero; the centres are positive)
        ix = np.clip(np.floor(np.asarray(x0) + 0.5).astype(np.int64) - 1, 0, mask.shape[0] - 1)
        iy = np.clip(np.floor(np.asarray(y0) + 0.5).astype(np.int64) - 1, 0, mask.shape[1] - 1)
        hole = ~mask[ix, iy].astype(bool)
        u = np.where(hole, np.nan, u)
        v = np.where(hole, np.nan, v)
    u, v, cc = funRemoveOutliers(u, v, cc, 0, 100, ctx=ctx)
    DICpara = dict(DICpara, InitFFTSearchMethod=method, SizeOfFFTSearchRegion=s)
    return DICpara, x0, y0, u, v, cc


def MeshSetUp(x, y, DICpara):
    """DICmesh = MeshSetUp(x, y, DICpara) (func/MeshSetUp.m), host bookkeeping as in the
    reference: the search grid x, y (nY x nX, as funIntegerSearch returns them) becomes the
    FE node list coordinatesFEM (XList fastest), the Q4 elements elementsFEM (1-based) and the
    world copies (y -> ImgSize(2) + 1 - y, the reference's choice of ImgSize(2)).  The
    reference also builds a cell-corner mesh that it never stores (func/MeshSetUp.m:44-61,
    its fields commented out at :82-83); it is left out.  Returns a dict with the
    reference's field names."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    img_n = DICpara["ImgSize"][1]          # ImgSize(2), func/MeshSetUp.m:88-89
    M, N = x.shape[1], x.shape[0]          # M along XList (image x), N along YList
    xt, yt = x.T, y.T                      # M x N
    coordinatesFEM = np.stack([xt.ravel(order="F"), yt.ravel(order="F")], 1)
    j, i = np.meshgrid(np.arange(1, N), np.arange(1, M), indexing="ij")
    j, i = j.ravel(), i.ravel()            # element order: i (XList) fastest
    elementsFEM = np.stack([(j - 1) * M + i, (j - 1) * M + i + 1, j * M + i + 1, j * M + i], 1)
    return {"coordinatesFEM": coordinatesFEM, "elementsFEM": elementsFEM,
            "dirichlet": [], "neumann": [], "x0": xt, "y0": yt, "M": M, "N": N,
            "y0World": img_n + 1 - yt,
            "coordinatesFEMWorld": np.stack([coordinatesFEM[:, 0], img_n + 1 - coordinatesFEM[:, 1]], 1)}


def _box_sums(mask):
    """Inclusive box sums over a 1-based (x, y) pixel box of a mask, from its integral image."""
    S = np.zeros((mask.shape[0] + 1, mask.shape[1] + 1))
    S[1:, 1:] = np.cumsum(np.cumsum(np.asarray(mask, dtype=np.float64), 0), 1)

    def box(x0, x1, y0, y1):  # MATLAB mask(x0:x1, y0:y1), 1-based inclusive
        return S[x1, y1] - S[x0 - 1, y1] - S[x1, y0 - 1] + S[x0 - 1, y0 - 1]

    return box


def GenerateQuadtreeMesh(U0, Df, fNormalizedMask, DICmesh, DICpara):
    """[DICmesh, DICpara, U0] = GenerateQuadtreeMesh(U0, Df, fNormalizedMask, DICmesh, DICpara)
    (func_quadtree/GenerateQuadtreeMesh.m), host bookkeeping as in the reference:
      * from the uniform mesh of MeshSetUp, elements whose pixel box meets both values of the
        mask (funMarkEdge: max - min > 0) and are larger than DICmesh['elementMinSize'] are
        split in four, pass after pass (:27-36); a split also splits any coarser neighbour of
        the split element, so that every edge carries at most one hanging node (the
        1-irregular rule of the red refinement QrefineR applies; QrefineR itself is not
        vendored with the reference, so its node and element numbering is not restated:
        existing nodes keep their numbers, new nodes follow in element order);
      * corners in the reference's order (:40-48: (xmin, ymin), (xmax, ymin), (xmax, ymax),
        (xmin, ymax)) and hanging nodes in slots 5-8 (right, top, left, bottom edge, :50-67);
      * elements whose box is less than half mask (funMarkInside, :70-71) are dropped; their
        nodes stay in coordinatesFEM;
      * the dirichlet set markCoordHoleEdge (:74-104): nodes of refined elements and of
        elements within 1.01 winstepsize of the mesh border, grown twice by element
        adjacency;
      * U0 carried to the new nodes by linear interpolation over the Delaunay triangulation of
        the finite old nodes (scatteredInterpolant 'linear', :110-117; outside their hull the
        nearest old node's value, where the reference extrapolates linearly).
    Returns (DICmesh, DICpara, U0) with elementsFEM n_el x 8 and irregular (edge ends,
    midpoint) rows."""
    from scipy.interpolate import LinearNDInterpolator, NearestNDInterpolator

    C0 = np.asarray(DICmesh["coordinatesFEM"], dtype=np.float64)
    mask = np.asarray(fNormalizedMask)
    minsize = float(np.ravel(DICmesh.get("elementMinSize", 0))[0])
    step = float(np.ravel(DICpara["winstepsize"])[0])
    xs, ys = np.unique(C0[:, 0]), np.unique(C0[:, 1])
    M, N = xs.size, ys.size
    if M * N != C0.shape[0] or M < 2 or N < 2:
        raise AldicError("GenerateQuadtreeMesh: DICmesh must be the uniform mesh of MeshSetUp")
    if not (np.allclose(np.diff(xs), xs[1] - xs[0]) and np.allclose(np.diff(ys), ys[1] - ys[0])):
        raise AldicError("GenerateQuadtreeMesh: the uniform mesh must have one spacing")
    hx, hy = xs[1] - xs[0], ys[1] - ys[0]
    binary = np.isin(mask, (0, 1)).all()
    box = _box_sums(mask != 0) if binary else None

    def cell_box(L, i, j):
        x0, y0 = xs[0] + i * hx / 2 ** L, ys[0] + j * hy / 2 ** L
        x1, y1 = x0 + hx / 2 ** L, y0 + hy / 2 ** L
        if not all(float(v).is_integer() for v in (x0, x1, y0, y1)):
            raise AldicError("GenerateQuadtreeMesh: a refined element has non-integer corners "
                             "(the reference indexes the mask with them); raise elementMinSize")
        return int(x0), int(x1), int(y0), int(y1)

    def mixed(L, i, j):
        x0, x1, y0, y1 = cell_box(L, i, j)
        if binary:
            sm = box(x0, x1, y0, y1)
            return 0 < sm < (x1 - x0 + 1) * (y1 - y0 + 1)
        blk = mask[x0 - 1:x1, y0 - 1:y1]
        return blk.max() - blk.min() > 0

    order = [(0, i, j) for j in range(N - 1) for i in range(M - 1)]  # MeshSetUp's element order
    leaves = set(order)

    def leaf_at(L, i, j):
        if i < 0 or j < 0 or i >= (M - 1) << L or j >= (N - 1) << L:
            return None
        for lv in range(L, -1, -1):
            key = (lv, i >> (L - lv), j >> (L - lv))
            if key in leaves:
                return key
        return None

    while True:
        marked = [c for c in order if min(hx, hy) / 2 ** c[0] > minsize and mixed(*c)]
        if not marked:
            break
        split = set(marked)
        queue = list(marked)
        while queue:
            L, i, j = queue.pop()
            for di, dj in ((1, 0), (0, 1), (-1, 0), (0, -1)):
                nb = leaf_at(L, i + di, j + dj)
                if nb is not None and nb[0] < L and nb not in split:
                    split.add(nb)
                    queue.append(nb)
        new_order = []
        for c in order:
            if c in split:
                L, i, j = c
                kids = [(L + 1, 2 * i, 2 * j), (L + 1, 2 * i + 1, 2 * j), (L + 1, 2 * i + 1, 2 * j + 1),
                        (L + 1, 2 * i, 2 * j + 1)]
                leaves.discard(c)
                leaves.update(kids)
                new_order.extend(kids)
            else:
                new_order.append(c)
        order = new_order
    # nodes: the uniform mesh's first, in its order; new corners in element order
    node = {(float(x), float(y)): k + 1 for k, (x, y) in enumerate(C0)}
    coords = [tuple(c) for c in C0]
    corners = []
    for L, i, j in order:
        x0, x1, y0, y1 = cell_box(L, i, j)
        ids = []
        for pt in ((x0, y0), (x1, y0), (x1, y1), (x0, y1)):
            pt = (float(pt[0]), float(pt[1]))
            if pt not in node:
                node[pt] = len(coords) + 1
                coords.append(pt)
            ids.append(node[pt])
        corners.append(ids)
    E = np.zeros((len(order), 8), dtype=np.int64)
    irregular = []
    for e, ((L, i, j), ids) in enumerate(zip(order, corners)):
        x0, x1, y0, y1 = cell_box(L, i, j)
        E[e, :4] = ids
        mids = (((x1, (y0 + y1) / 2), (ids[1], ids[2])), (((x0 + x1) / 2, y1), (ids[2], ids[3])),
                ((x0, (y0 + y1) / 2), (ids[3], ids[0])), (((x0 + x1) / 2, y0), (ids[0], ids[1])))
        for slot, (pt, ends) in enumerate(mids):
            k = node.get((float(pt[0]), float(pt[1])))
            if k is not None:
                E[e, 4 + slot] = k
                irregular.append((ends[0], ends[1], k))
    C = np.array(coords, dtype=np.float64)
    # funMarkInside: drop the elements whose box is less than half mask
    keep = []
    for e, (L, i, j) in enumerate(order):
        x0, x1, y0, y1 = cell_box(L, i, j)
        sm = box(x0, x1, y0, y1) if binary else float(mask[x0 - 1:x1, y0 - 1:y1].sum())
        keep.append(not sm < 0.5 * (x1 - x0) * (y1 - y0))
    E = E[np.array(keep, dtype=bool)]
    # the dirichlet set
    size = np.hypot(C[E[:, 0] - 1, 0] - C[E[:, 2] - 1, 0], C[E[:, 0] - 1, 1] - C[E[:, 2] - 1, 1])
    wsz = float(np.ravel(DICpara.get("winsize", 0))[0])
    mark = size < 0.99 * np.sqrt(2) * max(step, 0 * wsz)
    xMin, xMax, yMin, yMax = C0[:, 0].min(), C0[:, 0].max(), C0[:, 1].min(), C0[:, 1].max()
    mark |= C[E[:, 0] - 1, 0] < xMin + 1.01 * step
    mark |= C[E[:, 2] - 1, 0] > xMax - 1.01 * step
    mark |= C[E[:, 0] - 1, 1] < yMin + 1.01 * step
    mark |= C[E[:, 2] - 1, 1] > yMax - 1.01 * step

    def nodes_of(rows):
        u = np.unique(E[rows])
        return u[1:] if u.size and u[0] == 0 else u

    hole_edge = nodes_of(mark)
    for _ in range(2):
        rows = np.isin(E, hole_edge).any(1)
        hole_edge = nodes_of(rows)
    # U0 on the new nodes
    U0 = np.asarray(U0, dtype=np.float64).ravel()
    ok = np.flatnonzero(np.isfinite(U0[0::2]))
    Unew = np.zeros(2 * C.shape[0])
    if ok.size >= 3:
        for comp in (0, 1):
            vals = U0[2 * ok + comp]
            lin = LinearNDInterpolator(C0[ok], vals)(C)
            bad = ~np.isfinite(lin)
            if bad.any():
                lin[bad] = NearestNDInterpolator(C0[ok], vals)(C[bad])
            Unew[comp::2] = lin
    out = dict(DICmesh)
    out.update(coordinatesFEM=C, elementsFEM=E, irregular=np.array(irregular, dtype=np.int64).reshape(-1, 3),
               markCoordHoleEdge=hole_edge, dirichlet=hole_edge,
               coordinatesFEMWorld=np.stack([C[:, 0], mask.shape[1] + 1 - C[:, 1]], 1))
    return out, DICpara, Unew


def _fill_mask(Df, ImgRef):
    m = Df.get("ImgRefMask") if isinstance(Df, dict) else None
    return np.ones(np.shape(ImgRef)) if m is None else np.asarray(m)


def _load_frame(ctx, Df, ImgRef, ImgDef, mask):
    ctx.load_image(_lib.SLOT_REF, np.asarray(ImgRef, dtype=np.float64))
    ctx.load_image(_lib.SLOT_DEF, np.asarray(ImgDef, dtype=np.float64))
    ctx.set_mask(None if mask is None else np.asarray(mask, dtype=np.float64))
    ctx.set_gradients(np.asarray(Df["DfDx"], dtype=np.float64), np.asarray(Df["DfDy"], dtype=np.float64))


def bad_points_local(conv, rule="quadtree"):
    """Bad-point rules after the local IC-GN loop: codes < 0 or > 99 plus the iteration
    outlier test (func_quadtree/LocalICGNQuadtree.m:169-192: > max(mu + sigma, 6) with a
    normal fit; func/LocalICGN.m:170-182: > mean + 0.15 std).  Returns (bad index array,
    LocalICGNBadPtNum)."""
    conv = np.asarray(conv)
    n = conv.size
    bad = (conv < 0) | (conv > 99)
    row3 = int(np.sum(conv == 102))
    num = int(np.sum(bad)) - row3
    good = ~bad
    if rule == "quadtree":
        if good.sum() >= 3:
            mu = conv[good].mean()
            sd = conv[good].std(ddof=1)   # fitdist 'Normal' sigma (unbiased std)
        else:
            mu, sd = np.inf, 0.0
        thr = max(mu + sd, 6)
    else:
        mu = conv[good].mean() if good.any() else np.nan
        sd = conv[good].std(ddof=1) if good.sum() > 1 else np.nan
        thr = mu + 0.15 * sd
    bad = bad | (conv > thr)
    return np.nonzero(bad)[0], num if n else 0


def bad_points_subpb1(conv):
    """Subpb1Quadtree.m:130-143 rules: codes < 0 or > 99, plus > max(mean + 0.25 std, 10)."""
    conv = np.asarray(conv)
    bad = (conv < 0) | (conv > 99)
    row3 = int(np.sum(conv == 102))
    num = int(np.sum(bad)) - row3
    good = ~bad
    mu = conv[good].mean() if good.any() else np.nan
    sd = conv[good].std(ddof=1) if good.sum() > 1 else np.nan
    bad = bad | (conv > max(mu + 0.25 * sd, 10))
    return np.nonzero(bad)[0], num


def LocalICGN(U0, coordinatesFEM, Df, ImgRef, ImgDef, DICpara, ICGNmethod="GaussNewton", tol=1e-3,
              shapeFunctionOrder=1, ctx: Context | None = None, fill=True):
    """[U, F, HtempPar, LocalTime, ConvItPerEle, LocalICGNBadPtNum] = LocalICGN(...)
    (func/LocalICGN.m).  The device runs the loop body (:64-164); the bad-point marking
    (:166-189) follows; bad points are filled by natural-neighbour interpolation of the good
    ones (:198-220; outside their hull the nearest value, where MATLAB extrapolates
    linearly), or returned as NaN with fill=False."""
    if shapeFunctionOrder != 1:
        raise AldicError("only the first-order shape function is implemented (as in the reference)")
    ctx = ctx or default_context()
    _load_frame(ctx, Df, ImgRef, ImgDef, None)
    t0 = time.perf_counter()
    r = ctx.local_icgn(_lib.UNIFORM, np.asarray(coordinatesFEM, dtype=np.float64), U0, DICpara["winsize"], tol)
    local_time = time.perf_counter() - t0
    U, F, conv = r["U"].copy(), r["F"].copy(), r["conv"]
    bad, num = bad_points_local(conv, rule="uniform")
    U[2 * bad] = np.nan
    U[2 * bad + 1] = np.nan
    for k in range(4):
        F[4 * bad + k] = np.nan
    if fill:
        crd = np.asarray(coordinatesFEM, dtype=np.float64)
        nan_u = np.isnan(U[0::2])
        U = _fill.fill_nans_natural(crd, U.reshape(-1, 2), "nearest").ravel()
        F4 = F.reshape(-1, 4).copy()
        F4[nan_u] = np.nan  # F is filled over the same good nodes as U (:199-218)
        F = _fill.fill_nans_natural(crd, F4, "nearest").ravel()
    return U, F, r["H"], local_time, conv, num


def LocalICGNQuadtree(U0, coordinatesFEM, Df, ImgRef, ImgDef, DICpara, ICGNmethod="GaussNewton", tol=1e-3,
                      shapeFunctionOrder=1, ctx: Context | None = None, fill=True):
    """[U, F, HtempPar, LocalTime, ConvItPerEle, LocalICGNBadPtNum, markCoordHoleStrain]
    = LocalICGNQuadtree(...) (func_quadtree/LocalICGNQuadtree.m).  Device loop body
    (:67-164), then the bad-point rules (:167-202), then the fill of the bad displacements
    per connected region of Df['ImgRefMask'] and over the whole mesh (:208-325, natural
    neighbour with 'nearest' outside the hull; F keeps its NaN, as the reference's F fill is
    commented out); fill=False returns the bad points as NaN."""
    if shapeFunctionOrder != 1:
        raise AldicError("only the first-order shape function is implemented (as in the reference)")
    ctx = ctx or default_context()
    _load_frame(ctx, Df, ImgRef, ImgDef, Df.get("ImgRefMask"))
    t0 = time.perf_counter()
    r = ctx.local_icgn(_lib.QUADTREE, np.asarray(coordinatesFEM, dtype=np.float64), U0, DICpara["winsize"], tol)
    local_time = time.perf_counter() - t0
    U, F, conv = r["U"].copy(), r["F"].copy(), r["conv"]
    bad, num = bad_points_local(conv, rule="quadtree")
    U[2 * bad] = np.nan
    U[2 * bad + 1] = np.nan
    mark = np.nonzero(r["markHole"] == 1)[0]
    if fill:
        U = _fill.fill_quadtree(U, np.asarray(coordinatesFEM, dtype=np.float64), _fill_mask(Df, ImgRef))
    return U, F, r["H"], local_time, conv, num, mark


def Subpb1Quadtree(UOld, FOld, udual, vdual, coordinatesFEM, Df, ImgRef, ImgDef, mu, beta, HPar, ALSolveStep,
                   DICpara, ICGNmethod="GaussNewton", tol=1e-2, ctx: Context | None = None, fill=True):
    """[U, HPar, ALSub1Time, ConvItPerEle, LocalICGNBadPtNum] = Subpb1Quadtree(...)
    (func_quadtree/Subpb1Quadtree.m).  Device loop body (:71-126), then the bad-point rules
    (:130-149), then the region-wise and whole-mesh fill of the bad points (:188-254, the
    mask of DICpara['ImgRefMask']); fill=False returns them as NaN."""
    ctx = ctx or default_context()
    _load_frame(ctx, Df, ImgRef, ImgDef, Df.get("ImgRefMask"))
    n = np.asarray(coordinatesFEM).shape[0]
    wl = DICpara.get("winsize_List")
    if wl is None:
        wl = np.full((n, 2), DICpara["winsize"], dtype=np.int32)
    t0 = time.perf_counter()
    r = ctx.subpb1(_lib.QUADTREE, np.asarray(coordinatesFEM, dtype=np.float64), UOld, FOld, vdual, mu, tol,
                   winsize=int(DICpara["winsize"]), winsize_list=np.asarray(wl, dtype=np.int32))
    t = time.perf_counter() - t0
    U, conv = r["U"].copy(), r["conv"]
    bad, num = bad_points_subpb1(conv)
    U[2 * bad] = np.nan
    U[2 * bad + 1] = np.nan
    if fill:
        mask = DICpara.get("ImgRefMask")
        U = _fill.fill_quadtree(U, np.asarray(coordinatesFEM, dtype=np.float64),
                                np.ones(np.shape(ImgRef)) if mask is None else np.asarray(mask))
    return U, HPar, t, conv, num


def Subpb1(UOld, FOld, udual, vdual, coordinatesFEM, Df, ImgRef, ImgDef, mu, beta, HPar, ALSolveStep, DICpara,
           ICGNmethod="GaussNewton", tol=1e-2, ctx: Context | None = None, fill=True):
    """Uniform-mesh Subpb1 (func/Subpb1.m with func/funICGN_Subpb1.m); HPar is the n x 21
    Hessian array of LocalICGN (zeros at ALSolveStep 1, as the reference passes).  The bad
    points are marked NaN (:166-183) and, as the reference ends (:186-199), every node takes
    the gridfit 'springs' surface of the good ones (fill=False returns the marked field)."""
    ctx = ctx or default_context()
    _load_frame(ctx, Df, ImgRef, ImgDef, None)
    n = np.asarray(coordinatesFEM).shape[0]
    H = np.zeros((n, 21)) if (HPar is None or ALSolveStep <= 1) else np.asarray(HPar, dtype=np.float64)
    t0 = time.perf_counter()
    r = ctx.subpb1(_lib.UNIFORM, np.asarray(coordinatesFEM, dtype=np.float64), UOld, FOld, vdual, mu, tol,
                   winsize=int(DICpara["winsize"]), HPar=H)
    t = time.perf_counter() - t0
    U, conv = r["U"].copy(), r["conv"]
    bad, num = bad_points_subpb1(conv)
    U[2 * bad] = np.nan
    U[2 * bad + 1] = np.nan
    if fill:
        crd = np.asarray(coordinatesFEM, dtype=np.float64)
        xn, yn = np.unique(crd[:, 0]), np.unique(crd[:, 1])
        ii, jj = np.searchsorted(xn, crd[:, 0]), np.searchsorted(yn, crd[:, 1])
        for comp in (0, 1):
            zg = _fill.gridfit_springs(crd[:, 0], crd[:, 1], U[comp::2], xn, yn)
            U[comp::2] = zg[jj, ii]
    return U, HPar, t, conv, num


def epipolar_ICGN1(pointCandidate, Df, ImgRef, ImgDef, winsize, tol, ICGNmethod="GaussNewton",
                   ctx: Context | None = None):
    """ZNSSD = epipolar_ICGN1(pointCandidate, Df, ImgRef, ImgDef, winsize, tol)
    (func/epipolar_ICGN1.m), batched over the rows of pointCandidate (n x 2)."""
    ctx = ctx or default_context()
    _load_frame(ctx, Df, ImgRef, ImgDef, None)
    pts = np.atleast_2d(np.asarray(pointCandidate, dtype=np.float64))
    return ctx.epipolar_icgn(pts, winsize, tol)


def StereoMatch_STAQ(RD_L, RD_R, Normalized_L, Normalized_R, file_name_L, NormalizedMask_L, NormalizedMask_R,
                     DICpara, StereoInfo, stereoMatchShapeOrder=1, ctx: Context | None = None):
    """[StereoInfo, RD_L, RD_R] = StereoMatch_STAQ(...) (func/StereoMatch_STAQ.m), the stereo
    match of the first frame pair, step for step: gradients of the left image (:22), the
    whole-field search with its bad-point removal (IntegerSearchQuadtree, stereo distance,
    :25), the uniform mesh (MeshSetUp, :28) and Init (:33), nodes outside the left mask NaN
    (:36-41), the quadtree mesh (GenerateQuadtreeMesh with elementMinSize =
    DICpara['winsizeMin'], :63-64) and LocalICGNQuadtree with tol 1e-3 (:86-93), then
    ResultFEMesh_corr = coordinates + U (:105-117).  The search, Init and IC-GN run on the
    device; meshing and the fills on the host, as in the reference.  Only the first-order
    shape function exists (stereoMatchShapeOrder 1)."""
    if stereoMatchShapeOrder != 1:
        raise AldicError("StereoMatch_STAQ: only the first-order shape function is implemented")
    ctx = ctx or default_context()
    StereoInfo = dict(StereoInfo or {})
    RD_R = dict(RD_R or {})
    maskL = np.asarray(NormalizedMask_L, dtype=np.float64)
    Df = funImgGradient(Normalized_L, Normalized_L, maskL, ctx=ctx)
    DICpara, x0, y0, u, v, cc = IntegerSearchQuadtree(Normalized_L, Normalized_R, file_name_L, DICpara, -1, ctx=ctx)
    mesh = MeshSetUp(x0, y0, DICpara)
    U0 = Init(u, v, cc["max"], mesh["x0"], mesh["y0"], 0, ctx=ctx)
    C = mesh["coordinatesFEM"]
    ix = np.floor(C[:, 0] + 0.5).astype(np.int64) - 1
    iy = np.floor(C[:, 1] + 0.5).astype(np.int64) - 1
    out = maskL[ix, iy] < 1
    U0 = np.array(U0, dtype=np.float64)
    U0[2 * np.flatnonzero(out)] = np.nan
    U0[2 * np.flatnonzero(out) + 1] = np.nan
    StereoInfo["ResultFEMesh"] = {"coordinatesFEM": C, "elementsFEM": mesh["elementsFEM"],
                                  "winsize": DICpara["winsize"], "winstepsize": DICpara["winstepsize"],
                                  "gridxyROIRange": DICpara["gridxyROIRange"]}
    mesh["elementMinSize"] = DICpara["winsizeMin"]
    mesh, DICpara, U0 = GenerateQuadtreeMesh(U0, Df, maskL, mesh, DICpara)
    StereoInfo["ResultFEMeshEachFrame"] = {"coordinatesFEM": mesh["coordinatesFEM"],
                                           "elementsFEM": mesh["elementsFEM"],
                                           "markCoordHoleEdge": mesh["markCoordHoleEdge"]}
    U, *_ = LocalICGNQuadtree(U0, mesh["coordinatesFEM"], Df, Normalized_L, Normalized_R, DICpara, "GaussNewton",
                              1e-3, 1, ctx=ctx)
    StereoInfo["U"] = U
    Cq = mesh["coordinatesFEM"]
    StereoInfo["ResultFEMesh_corr"] = Cq + (U.reshape(-1, 2) if U.size == Cq.size else 0.0)
    RD_R["Coordinates_corr"] = StereoInfo["ResultFEMesh_corr"]
    StereoInfo["CalPointsNum"] = np.shape(u)
    return StereoInfo, RD_L, RD_R


def organizeMatchedPairds_quadtree_ST1(RD_L, RD_R, DICpara=None):
    """matchedPairs = organizeMatchedPairds_quadtree_ST1(RD_L, RD_R, DICpara)
    (func_quadtree/organizeMatchedPairds_quadtree_ST1.m:8-14): per frame the n x 4 pairs
    [xL yL xR yR], frame 1 the left mesh and its stereo match (RD_R['Coordinates_corr']),
    frame i + 1 both moved by their temporal displacements.  RD_L / RD_R hold
    ResultFEMeshEachFrame (a list whose first entry has coordinatesFEM), Coordinates_corr
    (right) and ResultDisp (a list of dicts with U, n x 2 or 2n interleaved)."""
    C = np.asarray(RD_L["ResultFEMeshEachFrame"][0]["coordinatesFEM"], dtype=np.float64)
    Cr = np.asarray(RD_R["Coordinates_corr"], dtype=np.float64)
    pairs = [np.concatenate([C, Cr], 1)]
    for dl, dr in zip(RD_L.get("ResultDisp", []), RD_R.get("ResultDisp", [])):
        ul = np.asarray(dl["U"], dtype=np.float64).reshape(-1, 2)
        ur = np.asarray(dr["U"], dtype=np.float64).reshape(-1, 2)
        pairs.append(np.concatenate([C + ul, Cr + ur], 1))
    return pairs


def _has_distortion(cameraParams, side):
    rad = np.ravel(cameraParams.get("radial" + side, [0.0, 0.0]))
    tan = np.ravel(cameraParams.get("tangential" + side, [0.0, 0.0]))
    return bool(np.any(rad != 0) or np.any(tan != 0))


def funUndistortPoints(matchedPairs, cameraParams, ctx: Context | None = None):
    """undistortedPoints = funUndistortPoints(matchedPairs, cameraParams)
    (func/funUndistortPoints.m): every frame's pairs [xL yL xR yR] (n x 4) with the left and
    right points undistorted by their camera's lens model.  cameraParams: dict with KL, KR
    (3x3) and radialL / tangentialL / radialR / tangentialR (absent = zero).  Rows with a
    non-finite entry come back NaN."""
    ctx = ctx or default_context()
    out = []
    for pts in matchedPairs:
        pts = np.asarray(pts, dtype=np.float64)
        res = np.full(pts.shape, np.nan)
        fin = np.all(np.isfinite(pts), axis=1)
        if fin.any():
            for side, cols in (("L", slice(0, 2)), ("R", slice(2, 4))):
                res[fin, cols] = ctx.undistort_points(pts[fin, cols], cameraParams["K" + side],
                                                      cameraParams.get("radial" + side, [0.0, 0.0]),
                                                      cameraParams.get("tangential" + side))
        out.append(res)
    return out


def stereoReconstruction_quadtree(matchedPairs, cameraParams, ctx: Context | None = None):
    """[FinalResult, reprojectionErrors] = stereoReconstruction_quadtree(matchedPairs, cameraParams)
    (func_quadtree/stereoReconstruction_quadtree.m).  matchedPairs: list of n x 4 arrays;
    cameraParams: dict with KL, KR (3x3), R (3x3), T (3,) and, optionally, the lens
    distortion (radialL, tangentialL, radialR, tangentialR): the points are undistorted
    first (funUndistortPoints) when any coefficient is non-zero."""
    ctx = ctx or default_context()
    if _has_distortion(cameraParams, "L") or _has_distortion(cameraParams, "R"):
        matchedPairs = funUndistortPoints(matchedPairs, cameraParams, ctx=ctx)
    coords, errs = [], []
    for pts in matchedPairs:
        xyz, err = ctx.triangulate(np.asarray(pts, dtype=np.float64), cameraParams["KL"], cameraParams["KR"],
                                   cameraParams["R"], cameraParams["T"])
        coords.append(xyz)
        errs.append(err)
    final = {"Coordinates": coords, "Displacement": [c - coords[0] for c in coords]}
    return final, errs
