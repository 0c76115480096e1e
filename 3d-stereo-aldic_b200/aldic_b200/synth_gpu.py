"""Seeded synthetic stereo frame sequences rendered on the GPU (torch).

The same analytic rendering as ``synth.render`` -- every speckle a Gaussian in material
(frame-0 plane) coordinates, splatted over a square window around its projected centre, each
pixel evaluated at its own material coordinates -- for image sizes and frame counts that a
numpy rendering would take minutes over.  Used only to make benchmark inputs.

``stereo_sequence``: the stereo rig of ``synth.stereo_pair`` (pinhole cameras, f px,
principal point at the image centre, baseline along world x, optical axes aimed at the plane
centre) looking at a speckled plane z = Z that is stretched progressively over the sequence
(uniaxial in x up to ``stretch`` at the last frame, lateral contraction ``poisson`` times
that in y) with a growing local out-of-plane bulge.  Frames are M x N uint16 images in the
library's layout (dim 1 = image x fastest), returned as flat CUDA tensors.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import synth


@dataclass
class SequenceScene:
    L: list            # per frame: flat uint16 CUDA tensor, M * N, x fastest
    R: list
    M: int
    N: int
    camL: synth.Camera
    camR: synth.Camera
    KL: np.ndarray     # 1-based pixel convention of the matched pairs
    KR: np.ndarray
    R_rl: np.ndarray
    T_rl: np.ndarray
    Z: float
    params: dict

    def material_to_world(self, X, Y, k):
        """World position (mm) of material point (X, Y) of the frame-0 plane at frame k (numpy)."""
        p = self.params
        s = p["stretch"] * k / max(p["frames"] - 1, 1)
        b = p["bulge"] * k / max(p["frames"] - 1, 1)
        w = b * np.exp(-((X - p["bulge_x"]) ** 2 + (Y - p["bulge_y"]) ** 2) / p["bulge_sigma"] ** 2)
        return np.stack([(1 + s) * X, (1 - p["poisson"] * s) * Y, self.Z + w], axis=-1)


def stereo_sequence(frames=50, M=4096, N=3000, seed=4, f=4000.0, baseline=300.0, Z=1000.0, plane_half=(640.0, 480.0),
                    density_px=0.0153, noise=2.0, amp=(60.0, 200.0), gain=200.0, stretch=0.08, poisson=0.3,
                    bulge=3.0, bulge_x=60.0, bulge_y=-40.0, bulge_sigma=80.0, device="cuda") -> SequenceScene:
    import torch

    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    yaw = math.degrees(math.atan(baseline / 2.0 / Z))
    K = np.array([[f, 0, (M + 1) / 2.0 - 1.0], [0, f, (N + 1) / 2.0 - 1.0], [0, 0, 1.0]])
    camL = synth.Camera(K=K, R=synth._rot_y(-yaw), C=np.array([-baseline / 2, 0.0, 0.0]))
    camR = synth.Camera(K=K, R=synth._rot_y(+yaw), C=np.array([+baseline / 2, 0.0, 0.0]))
    mm_per_px = Z / f
    hx, hy = plane_half
    n_sp = int(round(density_px * (2 * hx) * (2 * hy) / mm_per_px ** 2))
    sp = synth.make_speckles(rng, n_sp, -hx, hx, -hy, hy, 2.0 * mm_per_px, 4.0 * mm_per_px, amp[0], amp[1])
    params = dict(frames=frames, stretch=stretch, poisson=poisson, bulge=bulge, bulge_x=bulge_x, bulge_y=bulge_y,
                  bulge_sigma=bulge_sigma)
    f64 = dict(dtype=torch.float64, device=dev)
    cx, cy = torch.tensor(sp.cx, **f64), torch.tensor(sp.cy, **f64)
    ir2 = torch.tensor(1.0 / sp.r ** 2, **f64)
    aa = torch.tensor(sp.a * gain, **f64)
    # pixel grid, x fastest (the library's column-major M x N layout)
    Yg, Xg = torch.meshgrid(torch.arange(1, N + 1, **f64), torch.arange(1, M + 1, **f64), indexing="ij")
    Xg, Yg = Xg.reshape(-1), Yg.reshape(-1)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def deform(X, Y, k):
        s = stretch * k / max(frames - 1, 1)
        b = bulge * k / max(frames - 1, 1)
        w = b * torch.exp(-((X - bulge_x) ** 2 + (Y - bulge_y) ** 2) / bulge_sigma ** 2)
        return (1 + s) * X, (1 - poisson * s) * Y, Z + w, s, b

    def frame_img(cam, k):
        Kt, Rt, Ct = torch.tensor(cam.K, **f64), torch.tensor(cam.R, **f64), torch.tensor(cam.C, **f64)
        # speckle centres at frame k, projected (1-based pixel coordinates)
        Px, Py, Pz, s, b = deform(cx, cy, k)
        Xc = (torch.stack([Px, Py, Pz], 1) - Ct) @ Rt.T
        p = Xc @ Kt.T
        px, py = p[:, 0] / p[:, 2] + 1.0, p[:, 1] / p[:, 2] + 1.0
        # material coordinates of every pixel: ray / deformed-surface intersection by fixed point
        d = torch.stack([Xg - 1.0, Yg - 1.0, torch.ones_like(Xg)], 1) @ torch.linalg.inv(Kt).T @ Rt
        qx = torch.zeros_like(Xg)
        qy = torch.zeros_like(Xg)
        zt = torch.full_like(Xg, Z)
        for _ in range(8):
            t = (zt - Ct[2]) / d[:, 2]
            qx = (Ct[0] + t * d[:, 0]) / (1 + s)
            qy = (Ct[1] + t * d[:, 1]) / (1 - poisson * s)
            zt = Z + b * torch.exp(-((qx - bulge_x) ** 2 + (qy - bulge_y) ** 2) / bulge_sigma ** 2)
        del d
        img = torch.zeros(M * N, **f64)
        ipx, ipy = torch.round(px).long(), torch.round(py).long()
        keep = (ipx > -12) & (ipx <= M + 12) & (ipy > -12) & (ipy <= N + 12)
        ipx, ipy, kcx, kcy, kir2, ka = ipx[keep], ipy[keep], cx[keep], cy[keep], ir2[keep], aa[keep]
        offs = torch.arange(-12, 13, device=dev)
        Xp = ipx[:, None] + offs[None, :]            # all 25 window columns at once
        okx = (Xp >= 1) & (Xp <= M)
        for dy in range(-12, 13):
            Yp = ipy + dy
            ok = okx & ((Yp >= 1) & (Yp <= N))[:, None]
            lin = ((Xp - 1) + ((Yp - 1) * M)[:, None])[ok]
            sel = ok.nonzero()[:, 0]
            d2 = (qx[lin] - kcx[sel]) ** 2 + (qy[lin] - kcy[sel]) ** 2
            img.index_add_(0, lin, ka[sel] * torch.exp(-d2 * kir2[sel]))
        img += torch.randn(M * N, generator=gen, **f64) * (noise * gain)
        return torch.clamp(torch.round(img), 0, 65535).to(torch.int32).to(torch.uint16)

    Ls = [frame_img(camL, k) for k in range(frames)]
    Rs = [frame_img(camR, k) for k in range(frames)]
    R_rl = camR.R @ camL.R.T
    T_rl = -camR.R @ camR.C + R_rl @ (camL.R @ camL.C)
    K1 = np.array([[f, 0, (M + 1) / 2.0], [0, f, (N + 1) / 2.0], [0, 0, 1.0]])
    return SequenceScene(L=Ls, R=Rs, M=M, N=N, camL=camL, camR=camR, KL=K1, KR=K1, R_rl=R_rl, T_rl=T_rl, Z=Z,
                         params=params)


@dataclass
class FieldPair:
    ref: object        # flat uint8 CUDA tensor, M * N, x fastest
    deff: object
    M: int
    N: int
    field: "SmoothField"


class SmoothField:
    """u(x, y) = u0 + g_ux (x - xc) + g_uy (y - yc) + sum_k a_k sin(2 pi (kx_k x + ky_k y) + phi_k)
    (and v alike): a random offset, an optional random affine part (gradients up to `affine`
    about the centre (xc, yc)) and low-frequency sinusoids, scaled so that every displacement
    gradient stays <= gmax everywhere and, without the affine part, |u|, |v| <= umax (the
    bounds hold term by term)."""

    def __init__(self, rng, umax=12.0, gmax=0.05, waves=3, wl=(300.0, 1200.0), affine=0.0, centre=(0.0, 0.0)):
        off = rng.uniform(-0.5, 0.5, 2) * umax
        self.off = off
        self.centre = (float(centre[0]), float(centre[1]))
        self.lin = rng.uniform(-affine, affine, (2, 2)) if affine > 0 else np.zeros((2, 2))
        self.terms = []
        for comp in range(2):
            ts = []
            ru = umax - abs(off[comp])
            rg = gmax - np.abs(self.lin[comp]).max()
            for _ in range(waves):
                lam = rng.uniform(*wl)
                ang = rng.uniform(0, 2 * np.pi)
                kx, ky = np.cos(ang) / lam, np.sin(ang) / lam
                a = rng.uniform(0.3, 1.0) * min(ru / waves, rg / waves / (2 * np.pi / lam))
                ts.append((a, kx, ky, rng.uniform(0, 2 * np.pi)))
            self.terms.append(ts)

    def disp(self, x, y, xp=np):
        """(u, v) at (x, y) (1-based pixel coordinates; numpy or torch arrays via xp)."""
        out = []
        dx, dy = x - self.centre[0], y - self.centre[1]
        for comp in range(2):
            s = self.off[comp] + self.lin[comp, 0] * dx + self.lin[comp, 1] * dy
            for a, kx, ky, ph in self.terms[comp]:
                s = s + a * xp.sin(2 * np.pi * (kx * x + ky * y) + ph)
            out.append(s)
        return out[0], out[1]

    def grad(self, x, y):
        """[du/dx, dv/dx, du/dy, dv/dy] at (x, y) (numpy): the IC-GN gradient order."""
        g = {}
        for comp in range(2):
            gx = self.lin[comp, 0] + 0.0 * x
            gy = self.lin[comp, 1] + 0.0 * x
            for a, kx, ky, ph in self.terms[comp]:
                c = a * 2 * np.pi * np.cos(2 * np.pi * (kx * x + ky * y) + ph)
                gx = gx + c * kx
                gy = gy + c * ky
            g[comp] = (gx, gy)
        return np.stack([g[0][0], g[1][0], g[0][1], g[1][1]], -1)


def field_pair(seed, M=2048, N=2048, umax=12.0, gmax=0.05, density=0.0153, noise=2.0, device="cuda",
               affine=0.0) -> FieldPair:
    """A reference speckle image (Gaussian speckles r ~ U(2, 4) px, amplitude U(60, 200), as the
    other scenes) and the same speckle field carried by a SmoothField (affine part about the
    image centre), rendered analytically (every pixel evaluated at its own material
    coordinates, the inverse map by fixed point), uint8 with N(0, noise) noise."""
    import torch

    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    field = SmoothField(rng, umax, gmax, affine=affine, centre=((M + 1) / 2.0, (N + 1) / 2.0))
    n_sp = int(round(density * (M + 32) * (N + 32)))
    sp = synth.make_speckles(rng, n_sp, -16, M + 16, -16, N + 16, 2.0, 4.0, 60.0, 200.0)
    f64 = dict(dtype=torch.float64, device=dev)
    cx, cy = torch.tensor(sp.cx, **f64), torch.tensor(sp.cy, **f64)
    ir2 = torch.tensor(1.0 / sp.r ** 2, **f64)
    aa = torch.tensor(sp.a, **f64)
    Yg, Xg = torch.meshgrid(torch.arange(1, N + 1, **f64), torch.arange(1, M + 1, **f64), indexing="ij")
    Xg, Yg = Xg.reshape(-1), Yg.reshape(-1)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def render(px, py, qx, qy):
        img = torch.zeros(M * N, **f64)
        ipx, ipy = torch.round(px).long(), torch.round(py).long()
        keep = (ipx > -12) & (ipx <= M + 12) & (ipy > -12) & (ipy <= N + 12)
        ipx, ipy, kcx, kcy, kir2, ka = ipx[keep], ipy[keep], cx[keep], cy[keep], ir2[keep], aa[keep]
        offs = torch.arange(-12, 13, device=dev)
        Xp = ipx[:, None] + offs[None, :]
        okx = (Xp >= 1) & (Xp <= M)
        for dy in range(-12, 13):
            Yp = ipy + dy
            ok = okx & ((Yp >= 1) & (Yp <= N))[:, None]
            lin = ((Xp - 1) + ((Yp - 1) * M)[:, None])[ok]
            sel = ok.nonzero()[:, 0]
            d2 = (qx[lin] - kcx[sel]) ** 2 + (qy[lin] - kcy[sel]) ** 2
            img.index_add_(0, lin, ka[sel] * torch.exp(-d2 * kir2[sel]))
        img += torch.randn(M * N, generator=gen, **f64) * noise
        return torch.clamp(torch.round(img), 0, 255).to(torch.uint8)

    ref = render(cx, cy, Xg, Yg)
    fu, fv = field.disp(cx, cy, xp=torch)
    qx, qy = Xg.clone(), Yg.clone()
    for _ in range(30):  # material point of every deformed-image pixel: q = x - u(q)
        u, v = field.disp(qx, qy, xp=torch)
        qx, qy = Xg - u, Yg - v
    deff = render(cx + fu, cy + fv, qx, qy)
    return FieldPair(ref=ref, deff=deff, M=M, N=N, field=field)


class TileField:
    """A mosaic of independent affine warps: tile (i, j) (tile x tile pixels, 1-based rows
    i tile + 1 .. (i + 1) tile, columns alike) carries u(x) = U_ij + F_ij (x - c_ij) about its
    centre c_ij = (i tile + tile / 2 + 1, j tile + tile / 2 + 1)."""

    def __init__(self, U, F, tile):
        self.U, self.F, self.tile = U, F, tile  # (ti, tj, 2), (ti, tj, 4) [du/dx dv/dx du/dy dv/dy]

    def centres(self):
        """The tile centres, (2, n) float64 in tile order (i fastest)."""
        ti, tj = self.U.shape[:2]
        h = self.tile // 2 + 1
        X, Y = np.meshgrid(self.tile * np.arange(ti) + h, self.tile * np.arange(tj) + h, indexing="ij")
        return np.stack([X.ravel(order="F"), Y.ravel(order="F")], 0).astype(np.float64)

    def _at(self, x, y):
        i = ((np.asarray(x) - 1) // self.tile).astype(np.int64)
        j = ((np.asarray(y) - 1) // self.tile).astype(np.int64)
        h = self.tile // 2 + 1
        return i, j, x - (self.tile * i + h), y - (self.tile * j + h)

    def disp(self, x, y):
        i, j, dx, dy = self._at(x, y)
        U, F = self.U[i, j], self.F[i, j]
        return U[..., 0] + F[..., 0] * dx + F[..., 2] * dy, U[..., 1] + F[..., 1] * dx + F[..., 3] * dy

    def grad(self, x, y):
        i, j, _, _ = self._at(x, y)
        return self.F[i, j]


def tile_pair(seed, tiles=28, tile=72, umax=12.0, gmax=0.05, density=0.0153, noise=2.0, device="cuda") -> FieldPair:
    """Training pairs with an independent speckle pattern and affine warp per tile: a tiles x
    tiles mosaic of tile x tile pixels, tile (i, j) showing its own Gaussian speckles
    (r ~ U(2, 4) px, amplitude U(60, 200)) in the reference image and the same speckles under
    u = U + F (x - c) in the deformed image, U ~ U(-umax, umax)^2, F ~ U(-gmax, gmax)^4,
    rendered analytically (the exact inverse of the affine map per pixel), uint8 with
    N(0, noise) noise.  The tile x tile window about each tile centre (1-based tile start +
    tile / 2) is the tile itself."""
    import torch

    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    M = N = tiles * tile
    U = rng.uniform(-umax, umax, (tiles, tiles, 2))
    F = rng.uniform(-gmax, gmax, (tiles, tiles, 4))
    field = TileField(U, F, tile)
    h = tile // 2 + 1
    box = tile // 2 + 32  # material half-box covering the tile and its warped preimage
    n_t = int(round(density * (2 * box) ** 2))
    f64 = dict(dtype=torch.float64, device=dev)
    ti = np.repeat(np.arange(tiles), tiles)
    tj = np.tile(np.arange(tiles), tiles)
    x0 = torch.tensor(np.repeat(tile * ti + h, n_t), **f64)
    y0 = torch.tensor(np.repeat(tile * tj + h, n_t), **f64)
    cx = x0 + torch.tensor(rng.uniform(-box, box, x0.numel()), **f64)
    cy = y0 + torch.tensor(rng.uniform(-box, box, x0.numel()), **f64)
    ir2 = torch.tensor(1.0 / rng.uniform(2.0, 4.0, x0.numel()) ** 2, **f64)
    aa = torch.tensor(rng.uniform(60.0, 200.0, x0.numel()), **f64)
    Ut = torch.tensor(np.repeat(U[ti, tj], n_t, axis=0), **f64)
    Ft = torch.tensor(np.repeat(F[ti, tj], n_t, axis=0), **f64)
    # A = I + F (rows: u, v; columns: d/dx, d/dy) and its inverse, per speckle
    a11, a21, a12, a22 = 1 + Ft[:, 0], Ft[:, 1], Ft[:, 2], 1 + Ft[:, 3]
    det = a11 * a22 - a12 * a21
    i11, i12, i21, i22 = a22 / det, -a12 / det, -a21 / det, a11 / det
    lo_x, lo_y = x0 - (h - 1), y0 - (h - 1)  # the speckle's tile, 1-based inclusive
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    offs = torch.arange(-12, 13, device=dev)

    def render(deformed):
        img = torch.zeros(M * N, **f64)
        if deformed:
            px = x0 + Ut[:, 0] + a11 * (cx - x0) + a12 * (cy - y0)
            py = y0 + Ut[:, 1] + a21 * (cx - x0) + a22 * (cy - y0)
        else:
            px, py = cx, cy
        ipx, ipy = torch.round(px).long(), torch.round(py).long()
        Xp = ipx[:, None] + offs[None, :]
        okx = (Xp >= lo_x[:, None]) & (Xp < lo_x[:, None] + tile)
        for dy in range(-12, 13):
            Yp = ipy + dy
            ok = okx & ((Yp >= lo_y) & (Yp < lo_y + tile))[:, None]
            sel = ok.nonzero()[:, 0]
            X = Xp[ok].double()
            Y = Yp[sel].double()
            if deformed:
                rx, ry = X - x0[sel] - Ut[sel, 0], Y - y0[sel] - Ut[sel, 1]
                qx = x0[sel] + i11[sel] * rx + i12[sel] * ry
                qy = y0[sel] + i21[sel] * rx + i22[sel] * ry
            else:
                qx, qy = X, Y
            lin = (Xp[ok] - 1) + (Yp[sel] - 1) * M
            d2 = (qx - cx[sel]) ** 2 + (qy - cy[sel]) ** 2
            img.index_add_(0, lin, aa[sel] * torch.exp(-d2 * ir2[sel]))
        img += torch.randn(M * N, generator=gen, **f64) * noise
        return torch.clamp(torch.round(img), 0, 255).to(torch.uint8)

    pair = FieldPair(ref=render(False), deff=render(True), M=M, N=N, field=field)
    pair.nodes = field.centres()
    return pair
