"""Seeded synthetic speckle scenes rendered analytically.

Images use the reference's internal convention: a numpy array ``A[i, j]`` with dim 1
(``i``) the image x and dim 2 (``j``) the image y, 1-based pixel coordinate ``x = i + 1``.
Intensity at a point p is ``sum_k a_k exp(-|q(p) - c_k|^2 / r_k^2)`` where ``q`` maps the
pixel to the material (reference) coordinates of the speckle pattern, so every frame is an
exact rendering, not a resampling of another frame.

Scenes:
  * ``temporal_affine``: one camera, uniform affine map (the 512x512 uint8 case).
  * ``stereo_pair``: two pinhole cameras looking at a speckled plane, frame 0 and frame 1
    (plane translated and rotated), uint16.
  * ``plate_with_hole``: circular hole + edge notch mask, smooth analytic field plus a
    sinusoid, uint8.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Speckles:
    cx: np.ndarray
    cy: np.ndarray
    r: np.ndarray
    a: np.ndarray


def make_speckles(rng, n, x0, x1, y0, y1, rmin, rmax, amin, amax) -> Speckles:
    return Speckles(cx=rng.uniform(x0, x1, n), cy=rng.uniform(y0, y1, n), r=rng.uniform(rmin, rmax, n),
                    a=rng.uniform(amin, amax, n))


def render(M, N, sp: Speckles, centre_px, to_material, reach_px, background=0.0):
    """Splat every speckle onto an M x N image.

    centre_px: (px, py) 1-based pixel positions of each speckle centre in this image.
    to_material: callable (X, Y) -> (qx, qy) mapping 1-based pixel coordinates to the
        material coordinates in which ``sp`` is defined (vectorised); evaluated once on
        the whole pixel grid.
    reach_px: half-size of the square pixel window evaluated around each centre.
    """
    I, J = np.meshgrid(np.arange(1, M + 1, dtype=np.float64), np.arange(1, N + 1, dtype=np.float64), indexing="ij")
    qxm, qym = to_material(I.ravel(order="F"), J.ravel(order="F"))
    qxm = np.asarray(qxm, dtype=np.float64)
    qym = np.asarray(qym, dtype=np.float64)
    img = np.full(M * N, background, dtype=np.float64)
    px = np.rint(centre_px[0]).astype(np.int64)
    py = np.rint(centre_px[1]).astype(np.int64)
    keep = (px > -reach_px) & (px <= M + reach_px) & (py > -reach_px) & (py <= N + reach_px)
    px, py = px[keep], py[keep]
    cx, cy, ir2, a = sp.cx[keep], sp.cy[keep], 1.0 / sp.r[keep] ** 2, sp.a[keep]
    K = int(reach_px)
    for dy in range(-K, K + 1):
        Y = py + dy
        oky = (Y >= 1) & (Y <= N)
        for dx in range(-K, K + 1):
            X = px + dx
            ok = oky & (X >= 1) & (X <= M)
            if not ok.any():
                continue
            lin = (X[ok] - 1) + (Y[ok] - 1) * M
            d2 = (qxm[lin] - cx[ok]) ** 2 + (qym[lin] - cy[ok]) ** 2
            img += np.bincount(lin, weights=a[ok] * np.exp(-d2 * ir2[ok]), minlength=M * N)
    return img.reshape((M, N), order="F")


def quantize(img, rng, noise_sigma, bits):
    top = (1 << bits) - 1
    out = img + rng.normal(0.0, noise_sigma, img.shape) if noise_sigma > 0 else img
    out = np.clip(np.rint(out), 0, top)
    return out.astype(np.uint8 if bits == 8 else np.uint16)


# ---------------------------------------------------------------------------------
# Scene 1: one camera, uniform affine deformation
# ---------------------------------------------------------------------------------
@dataclass
class AffineScene:
    ref: np.ndarray
    deff: np.ndarray
    u0: float
    v0: float
    dudx: float
    dvdy: float
    xc: float
    yc: float

    def disp(self, x, y):
        """True displacement (u along dim 1, v along dim 2) at 1-based (x, y)."""
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        return self.u0 + self.dudx * (x - self.xc), self.v0 + self.dvdy * (y - self.yc)


def temporal_affine(seed=0, M=512, N=512, n_speckles=4000, u=3.37, v=-1.82, dudx=0.002, dvdy=-0.001,
                    noise=2.0, bits=8) -> AffineScene:
    """512x512 uint8, 4000 Gaussian speckles r~U(2,4), a~U(60,200), N(0, noise) noise;
    deformed frame = the same field under x -> x + u(x) with u = (u, v) + diag(dudx, dvdy)(x - c)."""
    rng = np.random.default_rng(seed)
    sp = make_speckles(rng, n_speckles, -8, M + 8, -8, N + 8, 2.0, 4.0, 60.0, 200.0)
    xc, yc = (M + 1) / 2.0, (N + 1) / 2.0
    ident = lambda X, Y: (X, Y)
    ref = render(M, N, sp, (sp.cx, sp.cy), ident, 12)
    fx = sp.cx + u + dudx * (sp.cx - xc)
    fy = sp.cy + v + dvdy * (sp.cy - yc)
    inv = lambda X, Y: (xc + (X - xc - u) / (1.0 + dudx), yc + (Y - yc - v) / (1.0 + dvdy))
    deff = render(M, N, sp, (fx, fy), inv, 12)
    return AffineScene(ref=quantize(ref, rng, noise, bits), deff=quantize(deff, rng, noise, bits), u0=u, v0=v,
                       dudx=dudx, dvdy=dvdy, xc=xc, yc=yc)


# ---------------------------------------------------------------------------------
# Scene 2: calibrated stereo pair looking at a speckled plane
# ---------------------------------------------------------------------------------
def _rot_y(deg):
    t = math.radians(deg)
    return np.array([[math.cos(t), 0, math.sin(t)], [0, 1, 0], [-math.sin(t), 0, math.cos(t)]])


def _rodrigues(axis, ang):
    k = np.asarray(axis, dtype=np.float64)
    k = k / np.linalg.norm(k)
    Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + math.sin(ang) * Kx + (1 - math.cos(ang)) * Kx @ Kx


@dataclass
class Camera:
    K: np.ndarray      # 3x3 intrinsics (pixel coords: col = image x, row = image y)
    R: np.ndarray      # world -> camera rotation
    C: np.ndarray      # camera centre in world (mm)

    def project(self, Xw):
        Xc = (Xw - self.C) @ self.R.T
        p = Xc @ self.K.T
        return p[:, 0] / p[:, 2], p[:, 1] / p[:, 2]


@dataclass
class StereoScene:
    L: list            # [frame0, frame1] uint16 images (reference convention arrays)
    R: list
    camL: Camera
    camR: Camera
    KL: np.ndarray
    KR: np.ndarray
    R_rl: np.ndarray   # rotation of the right camera relative to the left (P_R = K_R [R|T])
    T_rl: np.ndarray
    plane_R: np.ndarray   # frame-1 rigid motion of the plane: X1 = plane_R @ X0 + plane_t
    plane_t: np.ndarray
    Z: float

    def plane_point_left(self, x, y, frame=0):
        """World point (mm; to_left_camera_frame gives the left camera's coordinates) seen at
        left pixel (x, y) (1-based image x/y) on the plane of `frame`."""
        return _ray_plane(self.camL, np.asarray(x, float), np.asarray(y, float), self.Z,
                          None if frame == 0 else (self.plane_R, self.plane_t))


def _ray_plane(cam: Camera, x, y, Z, motion=None):
    """Intersect pixel rays with the plane z = Z (frame 0) or with its rigidly moved copy."""
    Kinv = np.linalg.inv(cam.K)
    d = np.stack([x - 1.0, y - 1.0, np.ones_like(x)], axis=-1) @ Kinv.T   # pixel centre at integer coords
    dw = d @ cam.R                                                           # camera -> world direction
    if motion is None:
        n = np.array([0.0, 0.0, 1.0])
        p0 = np.array([0.0, 0.0, Z])
    else:
        Rm, tm = motion
        n = Rm @ np.array([0.0, 0.0, 1.0])
        p0 = Rm @ np.array([0.0, 0.0, Z]) + tm
    s = ((p0 - cam.C) @ n) / (dw @ n)
    return cam.C + s[..., None] * dw


def stereo_pair(seed=1, size=2048, f=4000.0, baseline=300.0, Z=1000.0, yaw_deg=None, plane_half=320.0,
                density_px=0.0153, bits=16, noise=2.0, amp=(60.0, 200.0), gain=200.0,
                motion_t=(0.1, -0.05, 0.3), motion_rot=1e-3) -> StereoScene:
    """Two pinhole cameras (f px, principal point at the image centre), baseline along
    world x, each yawed toward the target; the plane z = Z carries a seeded speckle field.
    Frame 1 moves the plane rigidly (translation motion_t in mm, rotation motion_rot rad).

    yaw_deg=None aims both optical axes at the plane centre (atan(baseline/2/Z)).
    Speckle density is matched to the 512^2 case in pixels: ~density_px speckles per px^2
    at the plane's central magnification, radius 2-4 px."""
    rng = np.random.default_rng(seed)
    if yaw_deg is None:
        yaw_deg = math.degrees(math.atan(baseline / 2.0 / Z))
    c = (size + 1) / 2.0
    K = np.array([[f, 0, c - 1.0], [0, f, c - 1.0], [0, 0, 1.0]])
    # World frame = left camera's frame rotated by its yaw; cameras at x = -b/2, +b/2 (mm).
    # camera x axis = image x (dim 1), camera y axis = image y (dim 2), z forward.
    camL = Camera(K=K, R=_rot_y(-yaw_deg), C=np.array([-baseline / 2, 0.0, 0.0]))
    camR = Camera(K=K, R=_rot_y(+yaw_deg), C=np.array([+baseline / 2, 0.0, 0.0]))
    mm_per_px = Z / f
    area_mm2 = (2 * plane_half) ** 2
    n_sp = int(round(density_px * area_mm2 / mm_per_px ** 2))
    sp = make_speckles(rng, n_sp, -plane_half, plane_half, -plane_half, plane_half, 2.0 * mm_per_px,
                       4.0 * mm_per_px, amp[0], amp[1])
    sp.a = sp.a * gain  # uint16 dynamic range
    Rm = _rodrigues([0.3, -0.5, 0.8], motion_rot)
    tm = np.asarray(motion_t, dtype=np.float64)

    def frame_img(cam, motion):
        # speckle centres in world for this frame
        Xw = np.stack([sp.cx, sp.cy, np.full_like(sp.cx, Z)], axis=-1)
        if motion is not None:
            Xw = (Xw - 0.0) @ motion[0].T + motion[1]
        u, v = cam.project(Xw)
        px, py = u + 1.0, v + 1.0   # 1-based

        def to_mat(X, Y):
            W = _ray_plane(cam, X, Y, Z, motion)
            if motion is not None:
                W = (W - motion[1]) @ motion[0]   # back to frame-0 plane coordinates
            return W[:, 0], W[:, 1]

        img = render(size, size, sp, (px, py), to_mat, 12)
        return quantize(img, rng, noise * (gain if bits == 16 else 1.0), bits)

    L0 = frame_img(camL, None)
    R0 = frame_img(camR, None)
    L1 = frame_img(camL, (Rm, tm))
    R1 = frame_img(camR, (Rm, tm))
    # P_L = K[I|0] in the left camera frame; right camera relative to left.
    R_rl = camR.R @ camL.R.T
    T_rl = -camR.R @ camR.C + R_rl @ (camL.R @ camL.C)
    K1 = np.array([[f, 0, c], [0, f, c], [0, 0, 1.0]])   # 1-based pixel convention of the matched pairs
    return StereoScene(L=[L0, L1], R=[R0, R1], camL=camL, camR=camR, KL=K1, KR=K1, R_rl=R_rl, T_rl=T_rl,
                       plane_R=Rm, plane_t=tm, Z=Z)


def stereo_truth(scene: StereoScene, coords_left, frame=0):
    """True matches of left pixels `coords_left` (n x 2, 1-based x/y): the right-image
    point of frame 0, the left/right points of `frame`, and the 3D points xyz0 / xyz1 in world
    coordinates (to_left_camera_frame gives the left camera's, those of the triangulation)."""
    x = coords_left[:, 0]
    y = coords_left[:, 1]
    W0 = _ray_plane(scene.camL, x, y, scene.Z)
    uR, vR = scene.camR.project(W0)
    out = {"right0": np.stack([uR + 1.0, vR + 1.0], axis=1), "xyz0": W0}
    if frame:
        W1 = W0 @ scene.plane_R.T + scene.plane_t
        uL1, vL1 = scene.camL.project(W1)
        uR1, vR1 = scene.camR.project(W1)
        out.update(left1=np.stack([uL1 + 1.0, vL1 + 1.0], axis=1), right1=np.stack([uR1 + 1.0, vR1 + 1.0], axis=1),
                   xyz1=W1)
    return out


def to_left_camera_frame(scene: StereoScene, Xw):
    return (Xw - scene.camL.C) @ scene.camL.R.T


# ---------------------------------------------------------------------------------
# Scene 3: plate with a hole (masked, smooth non-affine field)
# ---------------------------------------------------------------------------------
@dataclass
class HoleScene:
    ref: np.ndarray
    deff: np.ndarray
    mask: np.ndarray
    disp: callable = field(repr=False)


def plate_with_hole(seed=2, size=2048, hole_r=300.0, peak=5.0, sin_amp=0.5, sin_wl=200.0, noise=2.0,
                    n_speckles=None) -> HoleScene:
    rng = np.random.default_rng(seed)
    M = N = size
    xc = yc = (size + 1) / 2.0
    if n_speckles is None:
        n_speckles = int(round(0.0153 * (M + 16) * (N + 16)))
    sp = make_speckles(rng, n_speckles, -8, M + 8, -8, N + 8, 2.0, 4.0, 60.0, 200.0)
    a = hole_r

    def disp(x, y):
        # Kirsch-type far-field plus hole perturbation (smooth, decays from the hole), scaled
        # to `peak` px, plus a sinusoid along x.
        dx = x - xc
        dy = y - yc
        r2 = dx * dx + dy * dy + 1e-9
        f = a * a / r2
        u = peak * (dx / size * 2.0) * (1.0 + 0.5 * f)
        v = -0.3 * peak * (dy / size * 2.0) * (1.0 - 0.5 * f)
        u = u + sin_amp * np.sin(2 * np.pi * y / sin_wl)
        return u, v

    ident = lambda X, Y: (X, Y)
    ref = render(M, N, sp, (sp.cx, sp.cy), ident, 12)
    fu, fv = disp(sp.cx, sp.cy)

    def inv(X, Y):
        qx, qy = X.copy(), Y.copy()
        for _ in range(30):
            u, v = disp(qx, qy)
            qx, qy = X - u, Y - v
        return qx, qy

    deff = render(M, N, sp, (sp.cx + fu, sp.cy + fv), inv, 12)
    I, J = np.meshgrid(np.arange(1, M + 1, dtype=np.float64), np.arange(1, N + 1, dtype=np.float64), indexing="ij")
    mask = ((I - xc) ** 2 + (J - yc) ** 2 > hole_r ** 2).astype(np.float64)
    # edge notch: a 40 px wide slot from the left edge to the hole
    mask[(np.abs(J - yc) < 20) & (I < xc)] = 0.0
    return HoleScene(ref=quantize(ref, rng, noise, 8), deff=quantize(deff, rng, noise, 8), mask=mask, disp=disp)
