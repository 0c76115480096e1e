"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import
this module, as the checker.  The product path (the CUDA library under
3d-stereo-aldic_b200/) never calls it.

Arrays follow the reference's MATLAB layouts: images are column-major M x N (numpy
``order='F'``), coordinates are 1-based, U is interleaved [u1 v1 ...], F is interleaved
[F11 F21 F12 F22 ...], H is n x 21.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build(force: bool = False) -> None:
    """Compile liboracle.so (and _ref/ when the reference sources are present)."""
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "aldic_oracle.cpp")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_interp.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp, C.c_long, _dp]
        L.orc_normalize.argtypes = [_dp, C.c_int, C.c_int, _ip, _ip, _dp, _dp]
        L.orc_gradient.argtypes = [_dp, C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        L.orc_local_icgn.argtypes = [C.c_int, _dp, _dp, C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_long, _dp,
                                     _dp, C.c_int, C.c_double, _dp, _dp, _dp, _ip, C.c_void_p, C.c_int]
        L.orc_local_icgn_guess.argtypes = [C.c_int, _dp, _dp, C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_long, _dp,
                                           _dp, C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp, _ip, C.c_void_p,
                                           C.c_int]
        L.orc_subpb1.argtypes = [C.c_int, _dp, _dp, C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_long, _dp, _dp,
                                 _dp, _dp, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double, _dp, _ip,
                                 C.c_int]
        L.orc_epipolar_icgn.argtypes = [_dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_long, _dp, C.c_int, C.c_double,
                                        _dp, _ip, C.c_int]
        L.orc_search_grid.argtypes = [_ip, _ip, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_integer_search.argtypes = [_dp, _dp, C.c_int, C.c_int, _ip, _ip, _ip, C.c_int, C.c_int, _dp, _dp,
                                         _dp, _dp, _dp, C.c_void_p, C.c_int]
        L.orc_search_list.argtypes = [_dp, _dp, C.c_int, C.c_int, _ip, C.c_int, C.c_int, C.c_long, _ip, _ip,
                                      C.c_int, _dp, C.c_int]
        L.orc_search_check.argtypes = [_dp, _dp, C.c_int, C.c_int, _ip, C.c_int, C.c_int, C.c_long, _ip, _ip,
                                       C.c_int, _dp, C.c_int]
        L.orc_findpeak.argtypes = [_dp, C.c_int, C.c_int, _dp]
        L.orc_normxcorr2.argtypes = [_dp, C.c_int, C.c_int, _dp, C.c_int, C.c_int, _dp]
        L.orc_normxcorr2.restype = C.c_int
        L.orc_bwselect.argtypes = [_up, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _up]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own ba_interp2_spline.cpp built under _ref/ (None if absent)."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref_interp.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_interp2.argtypes = [_dp, C.c_long, C.c_long, _dp, _dp, C.c_long, _dp]
        R.ref_interp2.restype = C.c_int
        _REF = R
    return _REF


def _f64(a):
    """Column-major image -> contiguous buffer in MATLAB memory order."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def _flat(a, dtype=np.float64):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).ravel())


def interp(F, X, Y):
    """ba_interp2_spline(F, X, Y): X is the dim-2 and Y the dim-1 coordinate (1-based)."""
    F = np.asarray(F, dtype=np.float64)
    M, N = F.shape
    X = _flat(X)
    Y = _flat(Y)
    out = np.empty_like(X)
    lib().orc_interp(_f64(F), M, N, X, Y, X.size, out)
    return out


def ref_interp(F, X, Y):
    R = ref_lib()
    if R is None:
        raise RuntimeError("reference interpolation library not built")
    F = np.asarray(F, dtype=np.float64)
    M, N = F.shape
    X = _flat(X)
    Y = _flat(Y)
    out = np.empty_like(X)
    if R.ref_interp2(_f64(F), M, N, X, Y, X.size, out) != 0:
        raise RuntimeError("reference MEX raised an error")
    return out


def normalize(img, gridx, gridy):
    img = np.asarray(img, dtype=np.float64)
    M, N = img.shape
    out = np.empty(M * N)
    ms = np.empty(2)
    lib().orc_normalize(_f64(img), M, N, _flat(gridx, np.int32), _flat(gridy, np.int32), out, ms)
    return out.reshape((M, N), order="F"), ms


def gradient(img, mask=None):
    img = np.asarray(img, dtype=np.float64)
    M, N = img.shape
    gx = np.empty((M - 6) * (N - 6))
    gy = np.empty_like(gx)
    mk = None if mask is None else _f64(mask)
    lib().orc_gradient(_f64(img), None if mk is None else mk.ctypes.data, M, N, gx, gy)
    return gx.reshape((M - 6, N - 6), order="F"), gy.reshape((M - 6, N - 6), order="F")


class Frame:
    """Reference/deformed images plus gradients, in the reference's layout."""

    def __init__(self, ref, deff, mask, dfdx, dfdy):
        ref = np.asarray(ref, dtype=np.float64)
        self.M, self.N = ref.shape
        self.ref = _f64(ref)
        self.deff = _f64(deff)
        self.mask = None if mask is None else _f64(mask)
        self.dfdx = _f64(dfdx)
        self.dfdy = _f64(dfdy)

    def _mask_ptr(self):
        return None if self.mask is None else self.mask.ctypes.data


def local_icgn(frame: Frame, coords, U0, winsize, tol, variant=1, nthreads=0, F0=None):
    """Loop body of LocalICGN (variant 0) / LocalICGNQuadtree (variant 1); F0 (4n) starts
    from [F0 U0] instead of the reference's [0 U0] (the learned initial guess)."""
    coords = np.asarray(coords, dtype=np.float64)
    n = coords.shape[0]
    U = np.empty(2 * n)
    F = np.empty(4 * n)
    H = np.empty(21 * n)
    conv = np.empty(n, dtype=np.int32)
    mark = np.zeros(n, dtype=np.uint8)
    f0 = None if F0 is None else _flat(F0)
    lib().orc_local_icgn_guess(variant, frame.ref, frame.deff, frame._mask_ptr(), frame.dfdx, frame.dfdy, frame.M,
                               frame.N, n, _f64(coords), _flat(U0), None if f0 is None else f0.ctypes.data,
                               int(winsize), float(tol), U, F, H, conv, mark.ctypes.data if variant == 1 else None,
                               nthreads)
    return dict(U=U, F=F, H=H.reshape((n, 21), order="F"), conv=conv, markHole=mark)


def subpb1(frame: Frame, coords, UOld, FOld, vdual, mu, tol, winsize=None, winsize_list=None, HPar=None,
           variant=1, nthreads=0):
    """Loop body of Subpb1 (variant 0) / Subpb1Quadtree (variant 1)."""
    coords = np.asarray(coords, dtype=np.float64)
    n = coords.shape[0]
    U = np.empty(2 * n)
    conv = np.empty(n, dtype=np.int32)
    wl = None
    if variant == 1:
        wl = np.ascontiguousarray(np.asarray(winsize_list, dtype=np.int32).ravel(order="F"))
    hp = None if HPar is None else _f64(HPar)
    lib().orc_subpb1(variant, frame.ref, frame.deff, frame._mask_ptr(), frame.dfdx, frame.dfdy, frame.M, frame.N, n,
                     _f64(coords), _flat(UOld), _flat(FOld), _flat(vdual), None if wl is None else wl.ctypes.data,
                     int(winsize or 0), None if hp is None else hp.ctypes.data, float(mu), float(tol), U, conv,
                     nthreads)
    return dict(U=U, conv=conv)


def epipolar_icgn(frame: Frame, pts, winsize, tol, nthreads=0):
    pts = np.asarray(pts, dtype=np.float64)
    n = pts.shape[0]
    z = np.empty(n)
    conv = np.empty(n, dtype=np.int32)
    lib().orc_epipolar_icgn(frame.ref, frame.deff, frame.dfdx, frame.dfdy, frame.M, frame.N, n, _f64(pts),
                            int(winsize), float(tol), z, conv, nthreads)
    return z, conv


def search_grid(gridx, gridy, winsize, step):
    nx = C.c_int()
    ny = C.c_int()
    lib().orc_search_grid(_flat(gridx, np.int32), _flat(gridy, np.int32), int(winsize), int(step), C.byref(nx),
                          C.byref(ny))
    return nx.value, ny.value


def integer_search(f, g, search, gridx, gridy, winsize, step, nthreads=0, want_qf=True):
    """funIntegerSearch(f, g, search, gridx, gridy, winsize, step, 0): returns x, y, u, v, phi, qf."""
    f = np.asarray(f, dtype=np.float64)
    M, N = f.shape
    nx, ny = search_grid(gridx, gridy, winsize, step)
    outs = [np.empty(nx * ny) for _ in range(5)]
    qf = np.empty(2 * nx * ny) if want_qf else None
    s = np.asarray(search, dtype=np.int32).ravel()
    if s.size == 1:
        s = np.array([s[0], s[0]], dtype=np.int32)
    lib().orc_integer_search(_f64(f), _f64(g), M, N, _flat(s, np.int32), _flat(gridx, np.int32),
                             _flat(gridy, np.int32), int(winsize), int(step), *outs,
                             None if qf is None else qf.ctypes.data, nthreads)
    x, y, u, v, phi = [o.reshape((ny, nx), order="F") for o in outs]
    return dict(x=x, y=y, u=u, v=v, phi=phi, qf=None if qf is None else qf.reshape((nx * ny, 2), order="F"))


def search_list(f, g, search, gridx_end, gridy_end, ii, jj, winsize, nthreads=0):
    """Selected subsets of funIntegerSearchWholeField: template top-lefts (ii, jj),
    gridx(end)/gridy(end) of the run they belong to.  Returns n x 5 [u v phi pce ppe]."""
    f = np.asarray(f, dtype=np.float64)
    M, N = f.shape
    ii = _flat(ii, np.int32)
    jj = _flat(jj, np.int32)
    s = np.asarray(search, dtype=np.int32).ravel()
    if s.size == 1:
        s = np.array([s[0], s[0]], dtype=np.int32)
    out = np.empty(5 * ii.size)
    lib().orc_search_list(_f64(f), _f64(g), M, N, _flat(s, np.int32), int(gridx_end), int(gridy_end), ii.size,
                          ii, jj, int(winsize), out, nthreads)
    return out.reshape(-1, 5)


def search_check(f, g, search, gridx_end, gridy_end, ii, jj, winsize, nthreads=0):
    """The subsets of search_list computed over the crop only (bit-identical u, v, phi; no
    q-factors), for whole-grid checks.  Returns n x 4 [u v phi margin], margin = the crop's
    largest NCC minus its second largest."""
    f = np.asarray(f, dtype=np.float64)
    M, N = f.shape
    ii = _flat(ii, np.int32)
    jj = _flat(jj, np.int32)
    s = np.asarray(search, dtype=np.int32).ravel()
    if s.size == 1:
        s = np.array([s[0], s[0]], dtype=np.int32)
    out = np.empty(4 * ii.size)
    lib().orc_search_check(_f64(f), _f64(g), M, N, _flat(s, np.int32), int(gridx_end), int(gridy_end), ii.size,
                           ii, jj, int(winsize), out, nthreads)
    return out.reshape(-1, 4)


def findpeak(f):
    f = np.asarray(f, dtype=np.float64)
    out = np.empty(3)
    lib().orc_findpeak(_f64(f), f.shape[0], f.shape[1], out)
    return out  # xpeak (column), ypeak (row), max_f


def normxcorr2(T, A):
    T = np.asarray(T, dtype=np.float64)
    A = np.asarray(A, dtype=np.float64)
    m, n = T.shape
    ma, na = A.shape
    out = np.empty((ma + m - 1) * (na + n - 1))
    if lib().orc_normxcorr2(_f64(T), m, n, _f64(A), ma, na, out) != 0:
        raise ValueError("normxcorr2: template larger than image or constant")
    return out.reshape((ma + m - 1, na + n - 1), order="F")


def bwselect(bw, r, c, conn):
    """Connected component containing the 0-based seed (r, c)."""
    bw = np.asarray(bw, dtype=np.uint8)
    rows, cols = bw.shape
    out = np.empty(rows * cols, dtype=np.uint8)
    lib().orc_bwselect(_flat(bw.ravel(order="F"), np.uint8), rows, cols, int(r), int(c), int(conn), out)
    return out.reshape((rows, cols), order="F")


def triangulate(pairs, KL, KR, R, T):
    """DLT triangulation (stereoReconstruction_quadtree.m:30-52 via MATLAB triangulate):
    P_L = K_L [I | 0], P_R = K_R [R | T]; per finite row the homogeneous 4x4 system is
    solved by SVD (smallest right singular vector).  Returns xyz (n x 3) and the mean
    reprojection error of the two views (NaN rows where the input is not finite)."""
    pairs = np.asarray(pairs, dtype=np.float64)
    PL = np.asarray(KL, dtype=np.float64) @ np.hstack([np.eye(3), np.zeros((3, 1))])
    PR = np.asarray(KR, dtype=np.float64) @ np.hstack([np.asarray(R, np.float64), np.asarray(T, np.float64).reshape(3, 1)])
    n = pairs.shape[0]
    xyz = np.full((n, 3), np.nan)
    err = np.full(n, np.nan)
    ok = np.all(np.isfinite(pairs), axis=1)
    p = pairs[ok]
    if p.size:
        A = np.stack([p[:, 0:1] * PL[2] - PL[0], p[:, 1:2] * PL[2] - PL[1],
                      p[:, 2:3] * PR[2] - PR[0], p[:, 3:4] * PR[2] - PR[1]], axis=1)
        _, _, Vt = np.linalg.svd(A)
        X = Vt[:, -1, :]
        X = X[:, :3] / X[:, 3:4]
        Xh = np.hstack([X, np.ones((X.shape[0], 1))])
        pl = Xh @ PL.T
        pr = Xh @ PR.T
        el = np.hypot(pl[:, 0] / pl[:, 2] - p[:, 0], pl[:, 1] / pl[:, 2] - p[:, 1])
        er = np.hypot(pr[:, 0] / pr[:, 2] - p[:, 2], pr[:, 1] / pr[:, 2] - p[:, 3])
        xyz[ok] = X
        err[ok] = 0.5 * (el + er)
    return xyz, err


def inpaint_nans4(A):
    """inpaint_nans(A, 4), the spring analogy (func/inpaint_nans.m:369-398): springs from
    every NaN entry to each in-grid horizontal / vertical neighbour (:375-381), duplicate
    springs removed (:384), knowns moved to the right-hand side (:394) and the NaN entries
    solved in the least-squares sense (:398; MATLAB's sparse QR, here the normal equations
    of the same full-rank system, solved directly).  Restated in numpy / scipy."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    flat = A.ravel(order="F").copy()
    nan = np.flatnonzero(np.isnan(flat))
    if nan.size == 0:
        return A.copy()
    r, c = nan % m, nan // m
    pairs = []
    for dr, dc in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        rr, cc = r + dr, c + dc
        ok = (rr >= 0) & (rr < m) & (cc >= 0) & (cc < n)
        pairs.append(np.stack([nan[ok], (rr + cc * m)[ok]], 1))
    P = np.unique(np.sort(np.concatenate(pairs), 1), axis=0)
    k = P.shape[0]
    S = sp.csr_matrix((np.tile([1.0, -1.0], k), (np.repeat(np.arange(k), 2), P.ravel())), shape=(k, m * n))
    known = np.flatnonzero(~np.isnan(flat))
    rhs = -(S[:, known] @ flat[known])
    Su = S[:, nan].tocsc()
    x = spla.spsolve((Su.T @ Su).tocsc(), Su.T @ rhs)
    flat[nan] = x
    return flat.reshape((m, n), order="F")


def _del4_rows(m, n, nodes):
    """Rows of inpaint_nans method 3's operator (func/inpaint_nans.m:257-321) for the listed
    linear nodes (0-based, column-major, m rows x n columns): (node, column, coefficient)
    triples summed over the four stencil sets exactly as the reference's sparse() calls
    add them -- del^4 (13 points) for rows and columns 3..end-2, the 5-point del^2 on the
    second / second-last row or column, and [1 -2 1] along the border rows and columns.  The
    columns are the reference's linear (column-major) offsets, wraps on 2-row grids included."""
    r = nodes % m + 1
    c = nodes // m + 1                      # 1-based, as the reference's tests
    trip = []

    def add(sel, offs, coefs):
        g = nodes[sel]
        for o, w in zip(offs, coefs):
            trip.append((g, g + o, np.full(g.size, float(w))))

    add((r >= 3) & (r <= m - 2) & (c >= 3) & (c <= n - 2),
        (-2 * m, -m - 1, -m, -m + 1, -2, -1, 0, 1, 2, m - 1, m, m + 1, 2 * m),
        (1, 2, -8, 2, 1, -8, 20, -8, 1, 2, -8, 2, 1))
    add((((r == 2) | (r == m - 1)) & (c >= 2) & (c <= n - 1)) | (((c == 2) | (c == n - 1)) & (r >= 2) & (r <= m - 1)),
        (-m, -1, 0, 1, m), (1, 1, -4, 1, 1))
    add(((r == 1) | (r == m)) & (c >= 2) & (c <= n - 1), (-m, 0, m), (1, -2, 1))
    add(((c == 1) | (c == n)) & (r >= 2) & (r <= m - 1), (-1, 0, 1), (1, -2, 1))
    if not trip:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
    return (np.concatenate([t[0] for t in trip]), np.concatenate([t[1] for t in trip]),
            np.concatenate([t[2] for t in trip]))


def inpaint_nans3(A):
    """inpaint_nans(A, 3) (func/inpaint_nans.m:255-325): the NaN entries and their
    neighbours under the 12-point del^4 template (identify_neighbors, :633-676) get the rows
    of _del4_rows; the knowns move to the right-hand side (:323), the rows touching a NaN
    column are kept (:324) and the NaN entries take the least-squares solution (:328,
    MATLAB's sparse QR; here a dense SVD least-squares solve of the same system, exact for
    the full-column-rank grids the tests use).  Restated in numpy / scipy."""
    import scipy.sparse as sp

    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    flat = A.ravel(order="F").copy()
    nan = np.flatnonzero(np.isnan(flat))
    if nan.size == 0:
        return A.copy()
    r, c = nan % m, nan // m
    talks = ((-2, 0), (-1, -1), (-1, 0), (-1, 1), (0, -2), (0, -1), (0, 1), (0, 2), (1, -1), (1, 0), (1, 1), (2, 0))
    nb = []
    for dr, dc in talks:
        rr, cc = r + dr, c + dc
        ok = (rr >= 0) & (rr < m) & (cc >= 0) & (cc < n)
        nb.append((rr + cc * m)[ok])
    nodes = np.union1d(nan, np.concatenate(nb))
    i, j, w = _del4_rows(m, n, nodes)
    if i.size and (j.min() < 0 or j.max() >= m * n):
        raise IndexError("inpaint_nans3: a stencil index leaves the grid (the reference's sparse() errors)")
    F = sp.csr_matrix((w, (i, j)), shape=(m * n, m * n))
    F.sum_duplicates()
    F.eliminate_zeros()
    known = np.flatnonzero(~np.isnan(flat))
    rhs = -(F[:, known] @ flat[known])
    Fn = F[:, nan].tocsr()
    k = np.flatnonzero(np.diff(Fn.indptr) > 0)
    x = np.linalg.lstsq(Fn[k].toarray(), rhs[k], rcond=None)[0]
    flat[nan] = x
    return flat.reshape((m, n), order="F")


def medfilt2_skip(V):
    """medFilt2(V, [2 2], 'symmetric', 2) of func/funRemoveOutliers.m:393-441 in MATLAB's
    single precision (the neighbour stack is single, :413): the median of V(r, c),
    V(r+1, c), V(r+1, c+1) with the last row and column repeated past the edge (the
    'post' symmetric pad of one, :403-409; neighbour 2 = V(r, c+1) is skipped, :426-431)."""
    V = np.asarray(V).astype(np.float32)
    P = np.pad(V, ((0, 1), (0, 1)), mode="symmetric")
    st = np.stack([P[:-1, :-1], P[1:, :-1], P[1:, 1:]], 2)
    return np.sort(st, 2)[:, :, 1]


def med_remove_outliers(u, epsilon=0.1):
    """funMedRemoveOutliers (func/funRemoveOutliers.m:374-390): the normalised median
    fluctuation |u - median| / (median(|u - median|) + epsilon) of the method-3 inpainted
    field, in single precision as MATLAB evaluates double op single."""
    uf = inpaint_nans3(u)
    med = medfilt2_skip(uf)
    fl = (uf.astype(np.float32) - med).astype(np.float32)
    res = medfilt2_skip(np.abs(fl))
    return med, np.abs(fl / (res + np.float32(epsilon))).astype(np.float32)


def remove_outliers(u, v, thr=100.0):
    """[u, v] = funRemoveOutliers(u, v, cc, 0, Thr0) with Thr0 > 0 (func/funRemoveOutliers.m:
    16, :44-87), the call IntegerSearchQuadtree makes (func_quadtree/IntegerSearchQuadtree.m:
    158-160): entries whose |normalised fluctuation| (u and v combined) exceeds Thr0 are
    set NaN, both grids are inpainted (method 4) and the original NaN holes (of u) are NaN
    again.  Returns (u, v, list of removed linear indices, 0-based column-major)."""
    u = np.asarray(u, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    hole = np.isnan(u)
    _, n1 = med_remove_outliers(u)
    _, n2 = med_remove_outliers(v)
    mag = np.sqrt((n1 * n1 + n2 * n2).astype(np.float32)).astype(np.float32)
    bad = mag > thr
    u2, v2 = u.copy(), v.copy()
    u2[bad] = np.nan
    v2[bad] = np.nan
    u2, v2 = inpaint_nans4(u2), inpaint_nans4(v2)
    u2[hole] = np.nan
    v2[hole] = np.nan
    return u2, v2, np.flatnonzero(bad.ravel(order="F"))


def _gauss_rule(order):
    """Gauss points and weights of func_quadtree/Subpb2Quadtree.m:60-77 (orders 4 and 5 with
    the file's rounded constants)."""
    if order == 2:
        return [-1 / np.sqrt(3), 1 / np.sqrt(3)], [1.0, 1.0]
    if order == 3:
        return [0.0, np.sqrt(3 / 5), -np.sqrt(3 / 5)], [8 / 9, 5 / 9, 5 / 9]
    if order == 4:
        return [0.339981, -0.339981, 0.861136, -0.861136], [0.652145, 0.652145, 0.347855, 0.347855]
    if order == 5:
        return [0.0, 0.538469, -0.538469, 0.90618, -0.90618], [0.568889, 0.478629, 0.478629, 0.236927, 0.236927]
    raise ValueError("Gauss point order must be 2..5")


def quadtree_shape(ksi, eta, present):
    """The 8-node quadtree element's shape functions and their (ksi, eta) derivatives
    (func_quadtree/Subpb2Quadtree.m:138-148 and the funDN* functions :343-396): corners 1-4,
    mid-side (hanging) nodes 5-8 switched on by `present` (4 flags); sign(0) = 0 as MATLAB's."""
    d5, d6, d7, d8 = (1.0 if f else 0.0 for f in present)
    sg = np.sign
    N5 = d5 * 0.5 * (1 + ksi) * (1 - abs(eta))
    N6 = d6 * 0.5 * (1 + eta) * (1 - abs(ksi))
    N7 = d7 * 0.5 * (1 - ksi) * (1 - abs(eta))
    N8 = d8 * 0.5 * (1 - eta) * (1 - abs(ksi))
    N = np.array([(1 - ksi) * (1 - eta) * 0.25 - 0.5 * (N7 + N8), (1 + ksi) * (1 - eta) * 0.25 - 0.5 * (N8 + N5),
                  (1 + ksi) * (1 + eta) * 0.25 - 0.5 * (N5 + N6), (1 - ksi) * (1 + eta) * 0.25 - 0.5 * (N6 + N7),
                  N5, N6, N7, N8])
    k5, e5 = d5 * 0.5 * (1 - abs(eta)), d5 * 0.5 * (1 + ksi) * sg(-eta)
    k6, e6 = d6 * 0.5 * (1 + eta) * sg(-ksi), d6 * 0.5 * (1 - abs(ksi))
    k7, e7 = d7 * 0.5 * (-1) * (1 - abs(eta)), d7 * 0.5 * (1 - ksi) * sg(-eta)
    k8, e8 = d8 * 0.5 * (1 - eta) * sg(-ksi), d8 * 0.5 * (-1) * (1 - abs(ksi))
    dk = np.array([-0.25 * (1 - eta) - 0.5 * (k7 + k8), 0.25 * (1 - eta) - 0.5 * (k8 + k5),
                   0.25 * (1 + eta) - 0.5 * (k5 + k6), -0.25 * (1 + eta) - 0.5 * (k6 + k7), k5, k6, k7, k8])
    de = np.array([-0.25 * (1 - ksi) - 0.5 * (e7 + e8), -0.25 * (1 + ksi) - 0.5 * (e8 + e5),
                   0.25 * (1 + ksi) - 0.5 * (e5 + e6), 0.25 * (1 - ksi) - 0.5 * (e6 + e7), e5, e6, e7, e8])
    return N, dk, de


def subpb2_element(xy, present, order, beta, mu, alpha):
    """Element matrices of Subpb2Quadtree (:149-204) for one element: xy (8 x 2, zeros at absent
    mid-side nodes, as the reference), returns the 16 x 16 element matrix
    sum_g |J| w ((beta + alpha) DN' DN + mu N' N) in the reference's dof order
    [x1 y1 x2 y2 ... x8 y8], and per Gauss point the data the right-hand side needs."""
    pts, wts = _gauss_rule(order)
    A = np.zeros((16, 16))
    gp = []
    for je, eta in enumerate(pts):          # ndgrid: ksi runs fastest
        for ik, ksi in enumerate(pts):
            w = wts[ik] * wts[je]
            N, dk, de = quadtree_shape(ksi, eta, present)
            J = np.array([[dk @ xy[:, 0], dk @ xy[:, 1]], [de @ xy[:, 0], de @ xy[:, 1]]])
            jac = J[0, 0] * J[1, 1] - J[0, 1] * J[1, 0]
            inv = np.array([[J[1, 1], -J[0, 1]], [-J[1, 0], J[0, 0]]]) / jac
            dx = inv[0, 0] * dk + inv[0, 1] * de
            dy = inv[1, 0] * dk + inv[1, 1] * de
            Nm = np.zeros((2, 16))
            Nm[0, 0::2], Nm[1, 1::2] = N, N
            DN = np.zeros((4, 16))
            DN[0, 0::2], DN[1, 0::2], DN[2, 1::2], DN[3, 1::2] = dx, dy, dx, dy
            A += jac * w * ((beta + alpha) * DN.T @ DN + mu * Nm.T @ Nm)
            gp.append((jac * w, Nm, DN))
    return A, gp


def subpb2_element_rhs(gp, beta, mu, alpha, ue, Fr):
    """Element right-hand side of Subpb2Quadtree (:203): sum_g |J| w (beta diag(DN' Fr') +
    mu N' N ue + alpha DN' DN ue); Fr holds, per dof row, the reference's F index row
    (F11, F12, F21, F22 of the dof's node)."""
    be = np.zeros(16)
    for jw, Nm, DN in gp:
        be += jw * (beta * np.einsum("ki,ik->i", DN, Fr) + mu * Nm.T @ Nm @ ue + alpha * DN.T @ DN @ ue)
    return be


def subpb2_quadtree(coords, elements, order, beta, mu, U, F, alpha=0.0, dirichlet=()):
    """[Uhat] = Subpb2Quadtree(DICmesh, GaussPtOrder, beta, mu, U, F, udual, vdual, alpha, ...)
    (func_quadtree/Subpb2Quadtree.m) with an empty neumann list: the element matrices and
    right-hand sides assembled element by element (:94-222; v and W are 0 * the duals,
    :40-41, so only U and F enter), the involved nodes all nodes of the elements but the
    first of unique(elementsFEM) (:234-238, the reference's way of dropping the 0 entry),
    the dirichlet nodes held at U (:271-273) and moved to the right-hand side, the free dofs
    solved directly (:276).  coords n x 2, elements n_el x 8 (1-based, 0 = no mid-side
    node), U 2n, F 4n; returns Uhat (2n; 0 at nodes neither free nor dirichlet)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    coords = np.asarray(coords, dtype=np.float64)
    E = np.asarray(elements, dtype=np.int64)
    n = coords.shape[0]
    U = np.asarray(U, dtype=np.float64).ravel()
    F = np.asarray(F, dtype=np.float64).ravel()
    rows, cols, vals = [], [], []
    b = np.zeros(2 * n)
    for e in range(E.shape[0]):
        ids = E[e, :8]
        present = [ids[k] != 0 for k in range(4, 8)]
        xy = np.zeros((8, 2))
        for k in range(8):
            if ids[k] != 0:
                xy[k] = coords[ids[k] - 1]
        A, gp = subpb2_element(xy, present, order, beta, mu, alpha)
        dof = np.full(16, -1)
        for k in range(8):
            if ids[k] != 0:
                dof[2 * k], dof[2 * k + 1] = 2 * (ids[k] - 1), 2 * (ids[k] - 1) + 1
        ue = np.array([U[d] if d >= 0 else 0.0 for d in dof])
        # the reference's F index rows: (F11, F12) for an x dof, (F21, F22) for a y dof
        Fr = np.zeros((16, 4))
        for k in range(8):
            if ids[k] != 0:
                a = ids[k] - 1
                Fr[2 * k] = Fr[2 * k + 1] = [F[4 * a], F[4 * a + 2], F[4 * a + 1], F[4 * a + 3]]
        be = subpb2_element_rhs(gp, beta, mu, alpha, ue, Fr)
        ok = dof >= 0
        ii, jj = np.meshgrid(dof[ok], dof[ok], indexing="ij")
        rows.append(ii.ravel())
        cols.append(jj.ravel())
        vals.append(A[np.ix_(ok, ok)].ravel())
        np.add.at(b, dof[ok], be[ok])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(2 * n, 2 * n))
    involved = np.unique(E[:, :8])[1:] - 1
    dnodes = np.unique(np.asarray(dirichlet, dtype=np.int64).ravel()) - 1 if np.size(dirichlet) else \
        np.zeros(0, np.int64)
    Uhat = np.zeros(2 * n)
    Uhat[2 * dnodes] = U[2 * dnodes]
    Uhat[2 * dnodes + 1] = U[2 * dnodes + 1]
    b = b - A @ Uhat
    fn = np.setdiff1d(involved, dnodes)
    free = np.sort(np.concatenate([2 * fn, 2 * fn + 1]))
    Uhat[free] = spla.spsolve(A[free][:, free].tocsc(), b[free])
    return Uhat


def _clip(poly, a, b):
    """Convex polygon (k x 2) clipped to the half-plane a . x <= b (Sutherland-Hodgman)."""
    out = []
    k = len(poly)
    for i in range(k):
        P, Q = poly[i], poly[(i + 1) % k]
        fp, fq = a @ P - b, a @ Q - b
        if fp <= 0:
            out.append(P)
        if (fp < 0 < fq) or (fq < 0 < fp):
            t = fp / (fp - fq)
            out.append(P + t * (Q - P))
    return np.array(out) if out else np.zeros((0, 2))


def _area(poly):
    if len(poly) < 3:
        return 0.0
    x, y = poly[:, 0], poly[:, 1]
    return 0.5 * abs(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1)))


def sibson_bruteforce(P, q):
    """Sibson (natural-neighbour) coordinates of q with respect to the points P (k x 2) by the
    definition, every point against every other: the Voronoi cell of q in P + {q}, and the
    part of it each old point's cell loses.  Returns (weights, bounded); bounded is False when
    q's cell is unbounded (q on or outside the convex hull).  For small tests only."""
    P = np.asarray(P, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    R0 = 4.0 * (np.abs(P - q).max() + 1.0)
    bounded = False
    for R in (R0, R0 * 64, R0 * 4096, R0 * 262144):  # a bounded cell stops touching a growing box
        V = q + R * np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=np.float64)
        for p in P:
            V = _clip(V, p - q, 0.5 * (p @ p - q @ q))
        if len(V) > 0 and np.abs(V - q).max() < 0.999 * R:
            bounded = True
            break
    w = np.zeros(len(P))
    for i, pi in enumerate(P):
        S = V
        for j, pj in enumerate(P):
            if j != i and len(S):
                S = _clip(S, pj - pi, 0.5 * (pj @ pj - pi @ pi))
        w[i] = _area(S)
    tot = w.sum()
    return (w / tot if tot > 0 else w), bounded


def _std8(vals):
    """MATLAB std(x, 'omitnan') of the listed values, summed in order (no fused operations)."""
    xs = [x for x in vals if not np.isnan(x)]
    k = len(xs)
    if k < 2:
        return 0.0 if k == 1 else np.nan
    m = 0.0
    for x in xs:
        m = m + x
    m = m / k
    ss = 0.0
    for x in xs:
        d = x - m
        ss = ss + d * d
    return np.sqrt(ss / (k - 1))


def spring_pass(u, v, mode):
    """One spring outlier pass of Init index 1 (func/Init.m:31-66, :76-109, :119-154): for every
    interior node of the inpainted grids, compare |value - neighbour average| with a multiple
    of the neighbours' standard deviation; a node failing the test for u or v is set NaN in
    both, with its neighbourhood; the border rows and columns are set NaN; both grids are
    inpainted again.  mode 0: 8 neighbours, weighted average (1/8 edge + 1/16 corner sums)
    / (3/4), 3 sigma, 8-neighbourhood; mode 1: 4 neighbours, plain mean, 2 sigma,
    4-neighbourhood; mode 2: as mode 0 with 2 sigma."""
    ut, vt = np.array(u, dtype=np.float64), np.array(v, dtype=np.float64)
    ui, vi = ut.copy(), vt.copy()
    m, n = ut.shape
    kk = 3.0 if mode == 0 else 2.0
    edge = ((-1, 0), (1, 0), (0, -1), (0, 1))
    corner = ((-1, -1), (1, -1), (1, 1), (-1, 1))
    for i in range(1, m - 1):
        for j in range(1, n - 1):
            bad = False
            for t in (ut, vt):
                e = [t[i + di, j + dj] for di, dj in edge]
                if mode == 1:
                    xs = [x for x in e if not np.isnan(x)]
                    avg = np.nan
                    if xs:
                        acc = 0.0
                        for x in xs:
                            acc = acc + x
                        avg = acc / len(xs)
                    sd = _std8(e)
                else:
                    c = [t[i + di, j + dj] for di, dj in corner]
                    se = ((e[0] + e[1]) + e[2]) + e[3]
                    sc = ((c[0] + c[1]) + c[2]) + c[3]
                    avg = ((1.0 / 8.0) * se + (1.0 / 16.0) * sc) / (3.0 / 4.0)
                    sd = _std8(e + c)
                err = abs(t[i, j] - avg) - kk * sd
                if err > 0:
                    bad = True
            if bad:
                nb = edge if mode == 1 else edge + corner
                for g in (ui, vi):
                    g[i, j] = np.nan
                    for di, dj in nb:
                        g[i + di, j + dj] = np.nan
    for g in (ui, vi):
        g[0, :] = np.nan
        g[-1, :] = np.nan
        g[:, 0] = np.nan
        g[:, -1] = np.nan
    return inpaint_nans4(ui), inpaint_nans4(vi)


def init_u0(u, v, index=0):
    """Init(u, v, Phi, x, y, index) (func/Init.m): inpaint_nans(., 4) of the search grids u, v
    (ny x nx) (:13), with index 1 the three spring outlier passes (:29-166), and U0 interleaved
    over the transposed grids (XList fastest) (:169-177)."""
    u, v = inpaint_nans4(u), inpaint_nans4(v)
    if index == 1:
        for mode in (0, 1, 2):
            u, v = spring_pass(u, v, mode)
    ui, vi = u.T.ravel(order="F"), v.T.ravel(order="F")
    U0 = np.empty(2 * ui.size)
    U0[0::2], U0[1::2] = ui, vi
    return U0


def distort_points(pts, K, radial, tangential=None):
    """The cameraParameters lens model (forward): undistorted pixels -> distorted pixels
    through normalised coordinates K^-1 (u, v, 1).  Used to check undistort_points."""
    K = np.asarray(K, dtype=np.float64)
    rad = list(np.ravel(radial)) + [0.0] * (3 - len(np.ravel(radial)))
    p1, p2 = (0.0, 0.0) if tangential is None else np.ravel(tangential)[:2]
    P = np.asarray(pts, dtype=np.float64).reshape(-1, 2)
    h = np.linalg.solve(K, np.stack([P[:, 0], P[:, 1], np.ones(len(P))]))
    x, y = h[0] / h[2], h[1] / h[2]
    r2 = x * x + y * y
    radial_f = 1.0 + r2 * (rad[0] + r2 * (rad[1] + r2 * rad[2]))
    xd = x * radial_f + 2 * p1 * x * y + p2 * (r2 + 2 * x * x)
    yd = y * radial_f + p1 * (r2 + 2 * y * y) + 2 * p2 * x * y
    q = K @ np.stack([xd, yd, np.ones_like(xd)])
    return np.stack([q[0] / q[2], q[1] / q[2]], 1)


def undistort_points(pts, K, radial, tangential=None):
    """MATLAB undistortPoints (func/funUndistortPoints.m:24-26) restated: the inverse of
    distort_points by fixed-point iteration x <- (xd - tangential(x)) / radial(x) in
    normalised coordinates, to 1e-15 (at most 200 steps).  Non-finite rows give NaN."""
    K = np.asarray(K, dtype=np.float64)
    rad = list(np.ravel(radial)) + [0.0] * (3 - len(np.ravel(radial)))
    p1, p2 = (0.0, 0.0) if tangential is None else np.ravel(tangential)[:2]
    P = np.asarray(pts, dtype=np.float64).reshape(-1, 2)
    out = np.full(P.shape, np.nan)
    fin = np.all(np.isfinite(P), axis=1)
    h = np.linalg.solve(K, np.stack([P[fin, 0], P[fin, 1], np.ones(int(fin.sum()))]))
    xd, yd = h[0] / h[2], h[1] / h[2]
    x, y = xd.copy(), yd.copy()
    for _ in range(200):
        r2 = x * x + y * y
        radial_f = 1.0 + r2 * (rad[0] + r2 * (rad[1] + r2 * rad[2]))
        tx = 2 * p1 * x * y + p2 * (r2 + 2 * x * x)
        ty = p1 * (r2 + 2 * y * y) + 2 * p2 * x * y
        xn, yn = (xd - tx) / radial_f, (yd - ty) / radial_f
        step = np.abs(xn - x) + np.abs(yn - y)
        x, y = xn, yn
        if np.all(step <= 1e-15 * (1.0 + np.abs(x) + np.abs(y))):
            break
    q = K @ np.stack([x, y, np.ones_like(x)])
    out[fin] = np.stack([q[0] / q[2], q[1] / q[2]], 1)
    return out
