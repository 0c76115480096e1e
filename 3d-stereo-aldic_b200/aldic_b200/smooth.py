"""The ALDIC loop's optional displacement smoothing, funSmoothDispQuadtree
(func_quadtree/funSmoothDispQuadtree.m), host code as in the reference: a regularised fit of
each displacement component on a lattice of spacing DICmesh['elementMinSize']
(regularizeNd, func/regularizeNd.m, in the two-dimensional 'linear' form the function
calls), a Gaussian filter that ignores NaN with edge correction (nanconv with 'edge' and
'nanout', func/nanconv.m), and the nodes read back from the lattice; two passes, as the
reference's loop runs (:45-64)."""
from __future__ import annotations

import numpy as np

from ._lib import AldicError


def regularize_2d(xy, z, xnodes, ynodes, smoothness):
    """yGrid = regularizeNd(xy, z, {xnodes, ynodes}, smoothness) with the defaults the drivers
    use ('linear' interpolation, the 'normal' solver): one fidelity row per point (bilinear
    weights of its lattice cell), and per axis one row per interior node of every lattice
    line with the three-point second-derivative weights 2 / ((x1 - x3)(x1 - x2)), ...,
    scaled by smoothness * sqrt(points / rows of that axis) * (axis range)^2; the normal
    equations solved directly.  Returns yGrid (len(xnodes) x len(ynodes)), yGrid[i, j] at
    (xnodes[i], ynodes[j])."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    xy = np.asarray(xy, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64).ravel()
    g = [np.asarray(xnodes, dtype=np.float64).ravel(), np.asarray(ynodes, dtype=np.float64).ravel()]
    n1, n2 = g[0].size, g[1].size
    if n1 < 3 or n2 < 3:
        raise AldicError("regularizeNd needs at least 3 lattice nodes per axis")
    if (xy[:, 0].min() < g[0][0] or xy[:, 0].max() > g[0][-1] or xy[:, 1].min() < g[1][0]
            or xy[:, 1].max() > g[1][-1]):
        raise AldicError("regularizeNd: all points must be within the range of the lattice")
    n = xy.shape[0]
    idx, frac = [], []
    for d in (0, 1):
        k = np.clip(np.searchsorted(g[d], xy[:, d], side="right") - 1, 0, g[d].size - 2)
        f = np.clip((xy[:, d] - g[d][k]) / np.diff(g[d])[k], 0, 1)
        idx.append(k)
        frac.append(f)
    rows, cols, vals = [], [], []
    for a, b in ((0, 0), (0, 1), (1, 0), (1, 1)):  # the cell's four nodes
        w = (frac[0] if a else 1 - frac[0]) * (frac[1] if b else 1 - frac[1])
        rows.append(np.arange(n))
        cols.append((idx[0] + a) + n1 * (idx[1] + b))
        vals.append(w)
    Afid = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n1 * n2))
    regs = []
    for d in (0, 1):
        x = g[d]
        x1, x2, x3 = x[:-2], x[1:-1], x[2:]
        w = 2.0 / np.stack([(x1 - x3) * (x1 - x2), (x2 - x1) * (x2 - x3), (x3 - x1) * (x3 - x2)], 1)
        if d == 0:
            ii, jj = np.meshgrid(np.arange(1, n1 - 1), np.arange(n2), indexing="ij")
            centre = (ii + n1 * jj).ravel(order="F")
            step = 1
            wd = w[(ii - 1).ravel(order="F")]
        else:
            ii, jj = np.meshgrid(np.arange(n1), np.arange(1, n2 - 1), indexing="ij")
            centre = (ii + n1 * jj).ravel(order="F")
            step = n1
            wd = w[(jj - 1).ravel(order="F")]
        m = centre.size
        scale = smoothness * np.sqrt(n / m) * (x[-1] - x[0]) ** 2
        regs.append(sp.csr_matrix((scale * wd.ravel(), (np.repeat(np.arange(m), 3),
                                                        np.stack([centre - step, centre, centre + step], 1).ravel())),
                                  shape=(m, n1 * n2)))
    A = sp.vstack([Afid] + regs).tocsc()
    rhs = np.concatenate([z, np.zeros(A.shape[0] - n)])
    sol = spla.spsolve((A.T @ A).tocsc(), A.T @ rhs)
    return sol.reshape((n1, n2), order="F")


def gaussian_kernel(size, std):
    """The rotationally symmetric Gaussian of fspecial('gaussian', size, std): exp(-(x^2 + y^2)
    / (2 std^2)) on the size x size stencil centred at 0, normalised to unit sum."""
    r = (size - 1) / 2.0
    x = np.arange(-r, r + 1)
    X, Y = np.meshgrid(x, x)
    h = np.exp(-(X * X + Y * Y) / (2.0 * std * std))
    return h / h.sum()


def nanconv_edge(a, k):
    """nanconv(a, k, 'edge', 'nanout') (func/nanconv.m): the 'same' convolution of a with NaN
    read as 0, divided by the convolution of the finite-entry indicator (edge correction),
    NaN where a was NaN."""
    from scipy.signal import convolve2d

    a = np.asarray(a, dtype=np.float64)
    nanm = np.isnan(a)
    a0 = np.where(nanm, 0.0, a)
    on = (~nanm).astype(np.float64)
    flat = convolve2d(on, k, mode="same")
    c = convolve2d(a0, k, mode="same") / flat
    c[nanm] = np.nan
    return c


def funSmoothDispQuadtree(U, DICmesh, DICpara):
    """U = funSmoothDispQuadtree(U, DICmesh, DICpara) (func_quadtree/funSmoothDispQuadtree.m):
    each component fitted by regularize_2d on the lattice min:h:max of the node coordinates
    (h = DICmesh['elementMinSize']; smoothness DICpara['DispSmoothness'], 5e-4 when absent),
    filtered by the Gaussian of DICpara['DispFilterStd'] (0 -> 0.5) and size
    DICpara['DispFilterSize'] (0 -> 2 ceil(2 std) + 1) with nanconv_edge, and read back at the
    nodes; two passes.  The reference prompts when the filter parameters are missing: here
    that raises.  Every node must lie on the lattice."""
    C = np.asarray(DICmesh["coordinatesFEM"], dtype=np.float64)
    h = float(np.ravel(DICmesh["elementMinSize"])[0])
    std = DICpara.get("DispFilterStd")
    size = DICpara.get("DispFilterSize")
    if std is None or size is None or np.size(std) == 0 or np.size(size) == 0:
        raise AldicError("funSmoothDispQuadtree: DispFilterStd and DispFilterSize are needed (the reference prompts)")
    std = float(std) or 0.5
    size = int(size) or int(2 * np.ceil(2 * std) + 1)
    smoothness = float(DICpara.get("DispSmoothness", 5e-4))
    xn = np.arange(C[:, 0].min(), C[:, 0].max() + h / 2, h)
    yn = np.arange(C[:, 1].min(), C[:, 1].max() + h / 2, h)
    ii = np.rint((C[:, 0] - xn[0]) / h).astype(np.int64)
    jj = np.rint((C[:, 1] - yn[0]) / h).astype(np.int64)
    if not (np.allclose(xn[ii], C[:, 0]) and np.allclose(yn[jj], C[:, 1])):
        raise AldicError("funSmoothDispQuadtree: a node is off the elementMinSize lattice")
    k = gaussian_kernel(size, std)
    U = np.array(U, dtype=np.float64).ravel()
    for _ in range(2):
        for comp in (0, 1):
            grid = regularize_2d(C, U[comp::2], xn, yn, smoothness)
            U[comp::2] = nanconv_edge(grid, k)[ii, jj]
    return U
