"""The drivers' fill of bad points after the local steps: MATLAB's scatteredInterpolant with
the 'natural' method (Sibson's natural-neighbour interpolation), host work in the reference
as here.

Callers in the reference: func/LocalICGN.m:199-220 (U, F over the whole mesh),
func_quadtree/LocalICGNQuadtree.m:212-247 (per connected region of the mask, 'natural' +
'nearest') and :300-325 (the whole mesh, 'natural' + 'nearest'),
func_quadtree/Subpb1Quadtree.m:193-254, func/TemporalMatch_quadtree_ST1.m:216-235 (F,
'natural' + 'none').

The per-query construction runs in the library's host code (aldic_sibson_weights); the
rare queries it hands back (cavities that reach the hull, ties that break the ring) take
the Python path below, and queries outside the hull the extrapolation.

Sibson coordinates of a query q with respect to the source points P are the shares of q's
Voronoi cell (in the diagram of P + {q}) that each old cell loses.  They are computed
exactly by half-plane clipping: the natural neighbours of q are the vertices of the Delaunay
triangles of P whose circumcircle holds q (the Bowyer-Watson cavity; a tolerance admits
circles through q, whose share is 0); q's cell is a box clipped by the bisectors of q and its
natural neighbours; each neighbour's share is that cell clipped by the bisectors of the
neighbour and its own Delaunay neighbours (which bound its old Voronoi cell).  A query whose
cell is unbounded lies on or outside the convex hull of P: on a hull edge it takes the
edge's linear interpolation (the limit of the Sibson coordinates there); outside, the value
of the nearest source ('nearest') or NaN ('none').  MATLAB's default 'linear'
extrapolation is not implemented (parity for queries outside the hull is unpinned)."""
from __future__ import annotations

import numpy as np

from ._lib import AldicError


class FillError(AldicError):
    """A bad argument to the natural-neighbour fill."""


def _clip(poly, a, b):
    """Convex polygon (k x 2) clipped to a . x <= b."""
    if len(poly) == 0:
        return poly
    f = poly @ a - b
    out = []
    k = len(poly)
    for i in range(k):
        j = (i + 1) % k
        if f[i] <= 0:
            out.append(poly[i])
        if (f[i] < 0 < f[j]) or (f[j] < 0 < f[i]):
            t = f[i] / (f[i] - f[j])
            out.append(poly[i] + t * (poly[j] - poly[i]))
    return np.array(out) if out else np.zeros((0, 2))


def _circumcentre(a, b, c):
    d = 2.0 * (a[0] * (b[1] - c[1]) + b[0] * (c[1] - a[1]) + c[0] * (a[1] - b[1]))
    a2, b2, c2 = a @ a, b @ b, c @ c
    return np.array([(a2 * (b[1] - c[1]) + b2 * (c[1] - a[1]) + c2 * (a[1] - b[1])) / d,
                     (a2 * (c[0] - b[0]) + b2 * (a[0] - c[0]) + c2 * (b[0] - a[0])) / d])


def _area(poly):
    if len(poly) < 3:
        return 0.0
    x, y = poly[:, 0], poly[:, 1]
    return 0.5 * abs(float(np.dot(x, np.roll(y, -1)) - np.dot(y, np.roll(x, -1))))


class NaturalNeighbor:
    """scatteredInterpolant(x, y, v, 'natural', extrap) over the source points P (k x 2)."""

    def __init__(self, P, extrapolation="nearest"):
        from scipy.spatial import Delaunay, cKDTree

        self.P = np.asarray(P, dtype=np.float64)
        if self.P.ndim != 2 or self.P.shape[1] != 2 or self.P.shape[0] < 3:
            raise FillError("natural-neighbour interpolation needs at least 3 source points (k x 2)")
        if extrapolation not in ("nearest", "none"):
            raise FillError("extrapolation must be 'nearest' or 'none'")
        self.extrap = extrapolation
        self.tri = Delaunay(self.P)
        self.kd = cKDTree(self.P)
        S = self.tri.simplices
        A, B, C = self.P[S[:, 0]], self.P[S[:, 1]], self.P[S[:, 2]]
        d = 2.0 * (A[:, 0] * (B[:, 1] - C[:, 1]) + B[:, 0] * (C[:, 1] - A[:, 1]) + C[:, 0] * (A[:, 1] - B[:, 1]))
        a2, b2, c2 = (A ** 2).sum(1), (B ** 2).sum(1), (C ** 2).sum(1)
        with np.errstate(divide="ignore", invalid="ignore"):
            ux = (a2 * (B[:, 1] - C[:, 1]) + b2 * (C[:, 1] - A[:, 1]) + c2 * (A[:, 1] - B[:, 1])) / d
            uy = (a2 * (C[:, 0] - B[:, 0]) + b2 * (A[:, 0] - C[:, 0]) + c2 * (B[:, 0] - A[:, 0])) / d
        self.cc = np.stack([ux, uy], 1)
        self.r2 = ((A - self.cc) ** 2).sum(1)
        self.nbr_ptr, self.nbr = self.tri.vertex_neighbor_vertices
        self.scale = float(np.ptp(self.P, axis=0).max()) or 1.0

    def _cavity(self, q):
        """Delaunay triangles whose circumcircle holds q (the query's simplex first), or None
        outside the hull."""
        s = int(self.tri.find_simplex(q))
        if s < 0:
            return None
        tol = 1e-10
        cav, seen, stack = [], {s}, [s]
        while stack:
            t = stack.pop()
            if ((q - self.cc[t]) ** 2).sum() <= self.r2[t] * (1 + tol) + (tol * self.scale) ** 2:
                cav.append(t)
                for u in self.tri.neighbors[t]:
                    if u >= 0 and u not in seen:
                        seen.add(u)
                        stack.append(u)
        return cav

    def weights(self, q):
        """(indices, Sibson weights) of the query q, or (None, None) when q's cell is unbounded.
        Watson's construction: walking the cavity's boundary around q, q's new Voronoi
        vertices are the circumcentres of (q, b_i, b_i+1); the area q takes from b_i is the
        polygon of the two new vertices at b_i and the circumcentres of the cavity triangles
        at b_i, in fan order.  Falls back to half-plane clipping when the cavity is not a
        simple ring (near-degenerate ties)."""
        q = np.asarray(q, dtype=np.float64)
        cav = self._cavity(q)
        if cav is None:
            return None, None
        S, NB = self.tri.simplices, self.tri.neighbors
        incav = set(cav)
        nxt, tri_of = {}, {}
        for t in cav:  # boundary edges, oriented counter-clockwise as the triangles are
            a, b, c = S[t]
            ccw = ((self.P[b] - self.P[a])[0] * (self.P[c] - self.P[a])[1]
                   - (self.P[b] - self.P[a])[1] * (self.P[c] - self.P[a])[0]) > 0
            for k in range(3):
                if NB[t][k] in incav:
                    continue
                if NB[t][k] < 0:
                    return self._weights_clip(q, cav)  # cavity reaches the hull
                u, v = S[t][(k + 1) % 3], S[t][(k + 2) % 3]
                if not ccw:
                    u, v = v, u
                if u in nxt:
                    return self._weights_clip(q, cav)
                nxt[u] = v
                tri_of[(u, v)] = t
        ring = [next(iter(nxt))]
        while True:
            w_ = nxt.get(ring[-1])
            if w_ is None:
                return self._weights_clip(q, cav)
            if w_ == ring[0]:
                break
            ring.append(w_)
            if len(ring) > len(nxt):
                return self._weights_clip(q, cav)
        if len(ring) != len(nxt):
            return self._weights_clip(q, cav)
        m = len(ring)
        B = self.P[ring]
        newv = np.array([_circumcentre(q, B[i], B[(i + 1) % m]) for i in range(m)])
        w = np.zeros(m)
        for i in range(m):
            bi = ring[i]
            prev, nx = ring[i - 1], ring[(i + 1) % m]
            t, came, end = tri_of[(prev, bi)], -1, tri_of[(bi, nx)]
            pts = [newv[i - 1]]
            for _ in range(len(cav) + 1):  # the fan of cavity triangles at bi
                pts.append(self.cc[t])
                if t == end:
                    break
                k_bi = int(np.nonzero(S[t] == bi)[0][0])
                step = -1
                for k in range(3):  # across an edge at bi, into the cavity, not back
                    u = NB[t][k]
                    if k != k_bi and u >= 0 and u in incav and u != came:
                        step = u
                        break
                if step < 0:
                    return self._weights_clip(q, cav)
                came, t = t, step
            else:
                return self._weights_clip(q, cav)
            pts.append(newv[i])
            w[i] = _area(np.array(pts))
        tot = w.sum()
        if not tot > 0:
            return None, None
        return np.array(ring), w / tot

    def _weights_clip(self, q, cav):
        """Sibson weights by clipping (see the module note); (None, None) for an unbounded cell."""
        nat = np.unique(self.tri.simplices[cav].ravel())
        # q's cell: a box clipped by the bisectors; a bounded cell stops touching the box as the
        # box grows (near the hull it can reach far past the neighbours), an unbounded one
        # never does
        R0 = 4.0 * (np.abs(self.P[nat] - q).max() + self.scale * 1e-6)
        V = None
        for R in (R0, R0 * 64, R0 * 4096, R0 * 262144):
            W = q + R * np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=np.float64)
            for i in nat:
                p = self.P[i]
                W = _clip(W, p - q, 0.5 * (p @ p - q @ q))
            if len(W) >= 3 and np.abs(W - q).max() < 0.999 * R:
                V = W
                break
        if V is None:
            return None, None  # on the hull or outside it
        w = np.zeros(len(nat))
        for k, i in enumerate(nat):
            pi = self.P[i]
            Sx = V
            for j in self.nbr[self.nbr_ptr[i]:self.nbr_ptr[i + 1]]:
                pj = self.P[j]
                Sx = _clip(Sx, pj - pi, 0.5 * (pj @ pj - pi @ pi))
                if len(Sx) == 0:
                    break
            w[k] = _area(Sx)
        tot = w.sum()
        if not tot > 0:
            return None, None
        return nat, w / tot

    def _on_hull_edge(self, q):
        """Linear interpolation weights along the hull edge that holds q, if one does."""
        tol = 1e-9 * self.scale
        for a, b in self.tri.convex_hull:
            pa, pb = self.P[a], self.P[b]
            e = pb - pa
            L2 = float(e @ e)
            t = float((q - pa) @ e) / L2
            if -1e-12 <= t <= 1 + 1e-12 and np.linalg.norm(pa + t * e - q) <= tol:
                return np.array([a, b]), np.array([1.0 - t, t])
        return None, None

    def native_weights(self, Q, cap=512):
        """Watson's construction for all queries at once in the library's host code
        (aldic_sibson_weights): (idx, w, count) with count -2 outside the hull and -1 where
        the construction needs the Python path."""
        import ctypes as C

        from . import _lib

        lib = _lib.load()
        Q = np.ascontiguousarray(np.atleast_2d(np.asarray(Q, dtype=np.float64)))
        m = Q.shape[0]
        P = np.ascontiguousarray(self.P)
        S = np.ascontiguousarray(self.tri.simplices, dtype=np.int32)
        NB = np.ascontiguousarray(self.tri.neighbors, dtype=np.int32)
        cc = np.ascontiguousarray(self.cc)
        r2 = np.ascontiguousarray(self.r2)
        qs = np.ascontiguousarray(self.tri.find_simplex(Q), dtype=np.int32)
        idx = np.zeros((m, cap), dtype=np.int32)
        w = np.zeros((m, cap))
        cnt = np.zeros(m, dtype=np.int32)
        vp = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
        rc = lib.aldic_sibson_weights(P.shape[0], vp(P), S.shape[0], vp(S), vp(NB), vp(cc), vp(r2), self.scale, m,
                                      vp(Q), vp(qs), cap, vp(idx), vp(w), vp(cnt))
        if rc != 0:
            raise FillError(f"aldic_sibson_weights failed with code {rc}")
        return idx, w, cnt

    def __call__(self, Q, V):
        """Values at the queries Q (m x 2) of the data V (k or k x c)."""
        Q = np.atleast_2d(np.asarray(Q, dtype=np.float64))
        V = np.asarray(V, dtype=np.float64)
        vec = V.ndim == 1
        V2 = V[:, None] if vec else V
        out = np.full((Q.shape[0], V2.shape[1]), np.nan)
        idx, w, cnt = self.native_weights(Q)
        for m, q in enumerate(Q):
            c = int(cnt[m])
            if c > 0:
                out[m] = w[m, :c] @ V2[idx[m, :c]]
                continue
            ii, ww = self.weights(q) if c == -1 else (None, None)
            if ii is None:
                ii, ww = self._on_hull_edge(q)
            if ii is not None:
                out[m] = ww @ V2[ii]
            elif self.extrap == "nearest":
                out[m] = V2[int(self.kd.query(q)[1])]
        return out[:, 0] if vec else out


def fill_nans_natural(coords, values, extrapolation="nearest"):
    """The reference's fill of one field over the mesh (func/LocalICGN.m:199-220, with
    'nearest' outside the hull): the rows of values (n x c) whose first column is NaN take
    the natural-neighbour interpolation of the finite rows.  Returns a filled copy."""
    coords = np.asarray(coords, dtype=np.float64)
    V = np.array(values, dtype=np.float64)
    bad = np.isnan(V[:, 0] if V.ndim > 1 else V)
    if not bad.any() or (~bad).sum() < 3:
        return V
    nn = NaturalNeighbor(coords[~bad], extrapolation)
    V[bad] = nn(coords[bad], V[~bad])
    return V


def fill_quadtree(U, coords, mask):
    """LocalICGNQuadtree's fill of NaN displacements (func_quadtree/LocalICGNQuadtree.m:
    212-247, then :300-325): per 8-connected region of the mask (bwconncomp), the region's NaN
    nodes from its finite nodes (a region with fewer than 3 skipped), by natural-neighbour
    interpolation with 'nearest' outside their hull; then whatever is still NaN from all
    finite nodes.  A node belongs to the region of its rounded pixel.  U: 2n interleaved (F is
    not filled there: the reference's F lines are commented out).  Returns a filled copy."""
    from scipy import ndimage

    coords = np.asarray(coords, dtype=np.float64)
    U2 = np.array(U, dtype=np.float64).reshape(-1, 2)
    mask = np.asarray(mask)
    bad = np.isnan(U2[:, 0])
    if bad.any():
        lab, nlab = ndimage.label(mask != 0, structure=np.ones((3, 3), dtype=int))
        ix = np.clip(np.floor(coords[:, 0] + 0.5).astype(np.int64) - 1, 0, mask.shape[0] - 1)
        iy = np.clip(np.floor(coords[:, 1] + 0.5).astype(np.int64) - 1, 0, mask.shape[1] - 1)
        node_lab = lab[ix, iy]
        for r in range(1, nlab + 1):
            inr = node_lab == r
            src = inr & ~bad
            qry = inr & bad
            if src.sum() < 3 or not qry.any():
                continue
            nn = NaturalNeighbor(coords[src], "nearest")
            U2[qry] = nn(coords[qry], U2[src])
        U2 = fill_nans_natural(coords, U2, "nearest")
    return U2.ravel()


def gridfit_springs(x, y, z, xnodes, ynodes, smoothness=1.0):
    """zgrid = gridfit(x, y, z, xnodes, ynodes, 'regularizer', 'springs') (func/gridfit.m,
    D'Errico's surface fit, vendored with the reference), the form func/Subpb1.m:189-190 calls:
    data points with a NaN dropped; each point's value tied to the grid by the 'triangle'
    interpolation of its cell (the diagonal from the cell's lower-left to its upper-right
    node); zero-rest-length springs between every node and its right, upper and two diagonal
    neighbours, stiffness 1 / (spacing / mean spacing) (autoscale); the spring rows scaled by
    smoothness * norm(A, 1) / norm(Areg, 1) under the data rows, and the stacked system
    solved in the least-squares sense (MATLAB's backslash; here its normal equations, which
    have the same solution for this full-rank system).  Returns zgrid (len(ynodes) x
    len(xnodes)), zgrid[j, i] at (xnodes[i], ynodes[j]).  The data must lie inside the node
    range (the reference's 'extend' case is not taken)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    x, y, z = (np.asarray(a, dtype=np.float64).ravel() for a in (x, y, z))
    keep = ~(np.isnan(x) | np.isnan(y) | np.isnan(z))
    x, y, z = x[keep], y[keep], z[keep]
    xn = np.asarray(xnodes, dtype=np.float64).ravel()
    yn = np.asarray(ynodes, dtype=np.float64).ravel()
    if x.min() < xn[0] or x.max() > xn[-1] or y.min() < yn[0] or y.max() > yn[-1]:
        raise FillError("gridfit: data outside the node range")
    nx, ny, n = xn.size, yn.size, x.size
    dx, dy = np.diff(xn), np.diff(yn)
    xscale, yscale = dx.mean(), dy.mean()
    # histc bins (0-based here), the last node folded into the last cell
    ix = np.clip(np.searchsorted(xn, x, side="right") - 1, 0, nx - 2)
    iy = np.clip(np.searchsorted(yn, y, side="right") - 1, 0, ny - 2)
    ind = iy + ny * ix  # column-major node index of the cell's lower-left node
    tx = np.clip((x - xn[ix]) / dx[ix], 0, 1)
    ty = np.clip((y - yn[iy]) / dy[iy], 0, 1)
    above = tx > ty
    L = np.where(above, ny, 1)
    t1, t2 = np.minimum(tx, ty), np.maximum(tx, ty)
    rows = np.repeat(np.arange(n), 3)
    cols = np.stack([ind, ind + ny + 1, ind + L], 1).ravel()
    vals = np.stack([1 - t2, t1, t2 - t1], 1).ravel()
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, nx * ny))
    blocks = []
    i, j = np.meshgrid(np.arange(nx), np.arange(ny - 1))          # springs along y
    k = (j + ny * i).ravel()
    st = 1.0 / (dy[j.ravel()] / yscale)
    blocks.append((k, k + 1, st))
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny))          # along x
    k = (j + ny * i).ravel()
    st = 1.0 / (dx[i.ravel()] / xscale)
    blocks.append((k, k + ny, st))
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1))      # the two diagonals
    k = (j + ny * i).ravel()
    st = 1.0 / np.sqrt((dx[i.ravel()] / xscale) ** 2 + (dy[j.ravel()] / yscale) ** 2)
    blocks.append((k, k + ny + 1, st))
    blocks.append((k + 1, k + ny, st))
    regs = []
    for a_, b_, st in blocks:
        m = a_.size
        regs.append(sp.csr_matrix((np.concatenate([-st, st]), (np.tile(np.arange(m), 2), np.concatenate([a_, b_]))),
                                  shape=(m, nx * ny)))
    Areg = sp.vstack(regs).tocsr()
    NA = abs(A).sum(0).max()
    NR = abs(Areg).sum(0).max()
    S = sp.vstack([A, Areg * (smoothness * NA / NR)]).tocsc()
    rhs = np.concatenate([z, np.zeros(Areg.shape[0])])
    zflat = spla.spsolve((S.T @ S).tocsc(), S.T @ rhs)
    return zflat.reshape((nx, ny)).T

