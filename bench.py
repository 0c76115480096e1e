#!/usr/bin/env python
"""Throughput of the ALDIC per-subset hot path on B200.

Metric: converged IC-GN subsets per second at <= 0.01 px from the FP64 oracle.

Workload (default ``learned2048``): the learned initial guess against the FFT integer search
on held-out 2048 x 2048 uint8 speckle frames (Gaussian speckles, a smooth random displacement
field with |u|, |v| <= 12 px and gradients <= 0.05, N(0, 2) noise), subset 33 (winsize 32),
step 16 (15 129 subsets per frame), tolerance 1e-3.  One step is one frame pair through one
path: load + normalise + gradients, then
  learned: network prediction -> IC-GN from [F0 U0] -> ZNCC check -> integer search (radius
           16) + IC-GN from [0 U0] on the subsets that failed (the fallback);
  fft:     whole-field integer search (radius 16) -> outlier removal -> Init -> IC-GN.
``value`` is the learned path, ``fft_init`` the FFT path on the same frames.

``stereo2048``: the calibrated stereo pair + temporal match + triangulation case -- two
synthetic pinhole cameras (f = 4000 px, principal point at the image centre, 300 mm baseline,
optical axes aimed at a speckled plane 1 m away), 2048 x 2048 uint16 frames 0 and 1 (plane
moved by (0.1, -0.05, 0.3) mm and a 1e-3 rad rotation), subset 41 (winsize 40), step 10 (~40k
subsets per camera); one step: prep (normalise 4 frames, gradients) -> stereo L0->R0 integer
search (search 70) + IC-GN (tol 1e-3) -> temporal L0->L1 and R0->R1 integer search (search 10)
+ IC-GN (tol 1e-2) -> FP64 triangulation of frames 0 and 1.
``temporal512`` is the single-camera 512 x 512 uint8 affine case (900 subsets).

A subset counts when the device flags it converged and its u, v are within 0.01 px of
the FP64 oracle run from the same initial guess on the same frames.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "3d-stereo-aldic_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# DRAM bytes (read + write) of one launch of the stereo search's correlation kernel, from an
# ncu capture of that launch (dram__bytes_read.sum + dram__bytes_write.sum, mean of four
# launches).  They are the inputs read about once each (frames, window map, ring tables).
TILE_TRAFFIC = {"stereo2048": 300_405_952, "stereo1024": 44_464_384}

METRIC = "converged IC-GN subsets/s at <=0.01 px vs FP64 oracle (FFT-search init), 1 B200"
UNIT = "subsets/s"


# ----------------------------------------------------------------------------------
# workload description
# ----------------------------------------------------------------------------------
def workload_params(name):
    if name == "learned2048":  # learned vs FFT initial guess, held-out 2048 x 2048 smooth-field frames
        return dict(size=2048, w=32, step=16, search=16, tol=1e-3, roi=20, umax=12.0, gmax=0.05, frames=8)
    if name == "learned1024":  # the same at 1024 x 1024 (profiling case)
        return dict(size=1024, w=32, step=16, search=16, tol=1e-3, roi=20, umax=12.0, gmax=0.05, frames=8)
    if name == "quadtree2048":
        return dict(size=2048, w=32, step=16, s_temp=10, tol_temp=1e-3, mu=1e-3, admm=2, min_elem=4)
    if name == "stereo2048":
        return dict(size=2048, w=40, step=10, s_stereo=70, s_temp=10, tol_stereo=1e-3, tol_temp=1e-2)
    if name == "stereo1024":  # same geometry at half the resolution (profiling case)
        return dict(size=1024, w=40, step=10, s_stereo=35, s_temp=10, tol_stereo=1e-3, tol_temp=1e-2)
    if name == "temporal512":
        return dict(size=512, w=30, step=16, s_temp=10, tol_temp=1e-3)
    if name == "sequence4096":  # 50 stereo frame pairs, 4096 x 3000 (x by y) uint16
        return dict(M=4096, N=3000, frames=50, w=40, step=10, s_stereo=(275, 375), s_temp=10, tol_stereo=1e-3,
                    tol_temp=1e-2, sample=64)
    raise SystemExit(f"unknown workload {name}")


def make_scene(name, seed):
    from aldic_b200 import synth

    if name == "stereo2048":
        return synth.stereo_pair(seed=seed, size=2048)
    if name == "stereo1024":
        return synth.stereo_pair(seed=seed, size=1024, f=2000.0)
    return synth.temporal_affine(seed=seed)


def grid_coords(M, N, w, step):
    """coordinatesFEM of the uniform mesh on the search grid (MeshSetUp ordering: XList fastest)."""
    xl = np.arange(1, M - w - step + 1, step)
    yl = np.arange(1, N - w - step + 1, step)
    X, Y = np.meshgrid(xl + w / 2.0, yl + w / 2.0, indexing="ij")
    return np.stack([X.ravel(order="F"), Y.ravel(order="F")], 1), len(xl), len(yl)


def crop_flops(M, N, w, step, s0, s1):
    """Algorithmic FLOPs of one whole-field search: 2 * (crop shifts) * (w+1)^2 per subset,
    with the reference's per-subset border clamps."""
    gx1, gy1 = M, N
    total = 0.0
    for ii in range(1, M - w - step + 1, step):
        L, R = s0, s1
        if ii - L < 1:
            L = ii - 1
        if ii + w + R > M:
            R = gx1 - ii - w - 1
        na = max(L, 0) + max(R, 0) + 3
        for jj in range(1, N - w - step + 1, step):
            U, D = s0, s1
            if jj - U < 1:
                U = jj - 1
            if jj + w + D > N:
                D = gy1 - jj - w - 1
            nb = max(U, 0) + max(D, 0) + 3
            total += 2.0 * na * nb * (w + 1) ** 2
    return total


def icgn_flops(conv, w):
    """Algorithmic FLOPs of one IC-GN call: 92 N per subset-iteration and 50 N once per subset
    that iterates (N = (w+1)^2); iterations = the code for converged subsets, 100 for code 101
    (max_iter reached or the warp left the image, counted as the full 100)."""
    conv = np.asarray(conv)
    it = np.where((conv > 0) & (conv <= 100), conv, np.where(conv == 101, 100, 0)).astype(np.float64)
    n_px = (w + 1) ** 2
    return float(92.0 * n_px * it.sum() + 50.0 * n_px * np.count_nonzero(it))


def tile_flops(M, N, w, step, s0, s1):
    """Algorithmic FLOPs of the shared-product correlation kernel for one whole-field search:
    2 per product f(x) g(x + d), formed once per tile position and shift (tiles of TI x 8
    grid subsets covering (TI-1)*step + w+1 rows by 7*step + w+1 columns, TI the most subset
    rows that fit 127 tile rows), over the (s0+s1+3)^2 shifts.  The block-sum additions and
    the NCC epilogue are not counted."""
    W1 = w + 1
    TI = (127 - W1) // step + 1
    FR, FC = (TI - 1) * step + W1, 7 * step + W1
    nx = len(range(1, M - w - step + 1, step))
    ny = len(range(1, N - w - step + 1, step))
    tiles = -(-nx // TI) * -(-ny // 8)
    nd = s0 + s1 + 3
    return 2.0 * FR * FC * nd * nd * tiles


# ----------------------------------------------------------------------------------
# clocks sampling during the timed region
# ----------------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, gpu_index):
        self.p = None
        self.path = os.path.join(tempfile.gettempdir(), f"aldic_clocks_{os.getpid()}.csv")
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={gpu_index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        rows = []
        try:
            with open(self.path) as fh:
                for line in fh:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 8:
                        rows.append(parts)
            os.remove(self.path)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[4 + i] and "Not" not in r[4 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------------
# the device pipeline
# ----------------------------------------------------------------------------------
class StereoPipeline:
    """Device-resident pass over one stereo frame set.  All work is enqueued on the
    current torch stream; no host synchronisation inside a step."""

    def __init__(self, A, torch, scene, P, device, autotune=True):
        self.A, self.torch, self.P, self.dev = A, torch, P, device
        self.icgn_events = None  # (start, stop) CUDA event pairs around the stereo IC-GN call
        M = N = P["size"]
        self.M, self.N = M, N
        self.coords_np, self.nx, self.ny = grid_coords(M, N, P["w"], P["step"])
        self.n = self.coords_np.shape[0]
        T = torch
        f64 = dict(dtype=T.float64, device=device)
        self.raw = {k: T.from_numpy(np.asfortranarray(img).ravel(order="F").copy()).to(device)
                    for k, img in (("L0", scene.L[0]), ("L1", scene.L[1]), ("R0", scene.R[0]), ("R1", scene.R[1]))}
        # MATLAB n x 2 column-major coordinatesFEM == a (2, n) row-major device tensor
        self.coords = T.from_numpy(np.ascontiguousarray(self.coords_np.T)).to(device)
        self.ctx = {k: A.Context(device.index or 0) for k in ("S", "L", "R")}
        # one stream per pass: the stereo pass owns the step's first and last work (the
        # timing stream); the temporal passes fork after the stereo search and join
        # before triangulation, so the stereo correlation kernel runs alone
        self.streams = {k: T.cuda.Stream(device) for k in ("S", "L", "R")}
        self.stream = self.streams["S"]
        for k, c in self.ctx.items():
            c.set_stream(self.streams[k].cuda_stream)
            # the first call of each call shape (a warm-up step) times the candidate kernel
            # configurations and keeps the fastest whose results agree
            c.set_option(A.OPT_AUTOTUNE, 1 if autotune else 0)
        self.ev = {k: T.cuda.Event() for k in ("fork", "S", "L", "R")}
        n, g = self.n, self.nx * self.ny
        # per pass: search grids, U0, the IC-GN results (U, F, codes; the per-subset Hessian
        # H feeds only ALDIC's Subpb1 step, which this pipeline does not run, so it is not
        # requested) and the grid-order Init output Ug
        self.buf = {}
        for k in ("S", "L", "R"):
            self.buf[k] = {"x": T.empty(g, **f64), "y": T.empty(g, **f64), "u": T.empty(g, **f64),
                           "v": T.empty(g, **f64), "phi": T.empty(g, **f64), "U0": T.empty(2 * n, **f64),
                           "U": T.empty(2 * n, **f64), "F": T.empty(4 * n, **f64),
                           "conv": T.empty(n, dtype=T.int32, device=device),
                           "mark": T.empty(n, dtype=T.uint8, device=device), "Ug": T.empty(2 * g, **f64),
                           "uo": T.empty(g, **f64), "vo": T.empty(g, **f64)}
        self.coordsR = T.empty((2, n), **f64)
        self.pairs = [T.empty((4, n), **f64), T.empty((4, n), **f64)]
        self.xyz = [{"xyz": T.empty(3 * n, **f64), "err": T.empty(n, **f64)} for _ in range(2)]
        self.KL, self.KR, self.Rm, self.Tv = scene.KL, scene.KR, scene.R_rl, scene.T_rl
        self.gx = [1, M]
        self.gy = [1, N]


    def _search_to_U0(self, b, ctx, out=None):
        """funRemoveOutliers(u, v, cc, 0, 100) (the end of IntegerSearchQuadtree), then
        Init(u, v, Phi, x, y, 0): the search grids (nY x nX column-major) inpainted
        (inpaint_nans(., 4)) and interleaved in mesh order, on the device."""
        # on copies (uo, vo): the raw search grids stay for the search parity check
        b["uo"].copy_(b["u"])
        b["vo"].copy_(b["v"])
        u, v = b["uo"].view(self.nx, self.ny), b["vo"].view(self.nx, self.ny)
        ctx.remove_outliers(u, v, 100.0)
        ctx.init_u0(u, v, out=b["U0"] if out is None else out)

    def step(self):
        T, st, ev = self.torch, self.streams, self.ev
        with T.cuda.stream(st["S"]):
            self._stereo_search()
        ev["fork"].record(st["S"])
        with T.cuda.stream(st["S"]):
            self._stereo_icgn()
        ev["S"].record(st["S"])
        with T.cuda.stream(st["L"]):
            st["L"].wait_event(ev["fork"])
            self._temporal_left()
        ev["L"].record(st["L"])
        with T.cuda.stream(st["R"]):
            st["R"].wait_event(ev["fork"])
            self._temporal_right(ev["S"])
        ev["R"].record(st["R"])
        with T.cuda.stream(st["S"]):
            st["S"].wait_event(ev["L"])
            st["S"].wait_event(ev["R"])
            self._triangulate()

    def _load_pair(self, c, ref, cur):
        shp = (self.M, self.N)
        c.load_image_raw(0, self.raw[ref], self.gx, self.gy, want_stats=False, shape=shp)
        c.load_image_raw(1, self.raw[cur], self.gx, self.gy, want_stats=False, shape=shp)
        c.compute_gradients()

    def _stereo_search(self):
        # stereo L0 -> R0
        P, cS, bS = self.P, self.ctx["S"], self.buf["S"]
        self._load_pair(cS, "L0", "R0")
        cS.integer_search([P["s_stereo"]] * 2, self.gx, self.gy, P["w"], P["step"], out=bS)

    def _stereo_icgn(self):
        P, bS = self.P, self.buf["S"]
        self._search_to_U0(bS, self.ctx["S"])
        ev = None
        if self.icgn_events is not None:  # on the launching stream, around the whole call
            T = self.torch
            ev = (T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True))
            ev[0].record(T.cuda.current_stream())
        self.ctx["S"].local_icgn(1, self.coords, bS["U0"], P["w"], P["tol_stereo"], out=bS)
        if ev is not None:
            ev[1].record(self.torch.cuda.current_stream())
            self.icgn_events.append(ev)

    def tuning(self):
        """The autotuner's choices of the three passes' contexts."""
        return {k: c.tuning_report() for k, c in self.ctx.items()}

    def _temporal_left(self):
        # temporal left L0 -> L1
        P, cL, bL = self.P, self.ctx["L"], self.buf["L"]
        self._load_pair(cL, "L0", "L1")
        cL.integer_search([P["s_temp"]] * 2, self.gx, self.gy, P["w"], P["step"], out=bL)
        self._search_to_U0(bL, cL)
        cL.local_icgn(1, self.coords, bL["U0"], P["w"], P["tol_temp"], out=bL)

    def _temporal_right(self, stereo_done):
        # temporal right R0 -> R1 on the stereo-matched mesh (coords + U_stereo)
        self._right_search()
        self.torch.cuda.current_stream().wait_event(stereo_done)
        self._right_icgn()

    def _right_search(self):
        P, cR = self.P, self.ctx["R"]
        self._load_pair(cR, "R0", "R1")
        cR.integer_search([P["s_temp"]] * 2, self.gx, self.gy, P["w"], P["step"], out=self.buf["R"])

    def _right_icgn(self):
        T, P = self.torch, self.P
        w, st = P["w"], P["step"]
        cR, bR, bS = self.ctx["R"], self.buf["R"], self.buf["S"]
        n = self.n
        US = bS["U"].view(n, 2)
        cxy = self.coords.t()
        xyR = cxy + T.nan_to_num(US, nan=0.0)
        self.coordsR.copy_(xyR.t())
        # Init over the search grid, then each right-image point takes its nearest grid node
        # (the MeshSetUp stand-in for the stereo-matched mesh)
        self._search_to_U0(bR, cR, out=bR["Ug"])
        i = T.clamp(T.round((xyR[:, 0] - (1 + w / 2.0)) / st), 0, self.nx - 1).long()
        j = T.clamp(T.round((xyR[:, 1] - (1 + w / 2.0)) / st), 0, self.ny - 1).long()
        bR["U0"].view(n, 2).copy_(bR["Ug"].view(-1, 2)[i + j * self.nx])
        cR.local_icgn(1, self.coordsR, bR["U0"], w, P["tol_temp"], out=bR)

    def _triangulate(self):
        # triangulation of frames 0 and 1
        T, n, cS = self.torch, self.n, self.ctx["S"]
        cxy = self.coords.t()
        US = self.buf["S"]["U"].view(n, 2)
        UL = self.buf["L"]["U"].view(n, 2)
        UR = self.buf["R"]["U"].view(n, 2)
        p0 = T.cat([cxy, cxy + US], 1)
        p1 = T.cat([cxy + UL, cxy + US + UR], 1)
        self.pairs[0].copy_(p0.t())
        self.pairs[1].copy_(p1.t())
        for k in range(2):
            cS.triangulate(self.pairs[k], self.KL, self.KR, self.Rm, self.Tv, out=self.xyz[k])

    def launches(self):
        return sum(c.launches for c in self.ctx.values())

    def close(self):
        for c in self.ctx.values():
            c.close()


# ----------------------------------------------------------------------------------
# verification against the FP64 oracle
# ----------------------------------------------------------------------------------
def oracle_frames(scene, P):
    import oracle as O

    M = N = P["size"]
    out = {}
    for key, img in (("L0", scene.L[0]), ("L1", scene.L[1]), ("R0", scene.R[0]), ("R1", scene.R[1])):
        out[key], _ = O.normalize(img.astype(np.float64), [1, M], [1, N])
    out["gL0"] = O.gradient(out["L0"])
    out["gR0"] = O.gradient(out["R0"])
    return out


def search_parity(dev_u, dev_v, ref, margin_tol=1e-6):
    """Integer-search parity over a whole grid: device u, v (grid order) against the oracle's
    search_check rows [u v phi margin].  A subset counts as exact when u and v are equal (or
    both NaN); a differing subset whose oracle peak margin is below margin_tol is a near-tie
    (the FP32 correlation cannot rank it), any other difference is a mismatch."""
    ou, ov, margin = ref[:, 0], ref[:, 1], ref[:, 3]
    same = ((dev_u == ou) & (dev_v == ov)) | (np.isnan(dev_u) & np.isnan(ou))
    tie = ~same & (margin < margin_tol)
    decided = margin >= margin_tol
    return {"search_exact": f"{int(same.sum())}/{same.size}",
            "search_exact_where_margin_ge_1e-6": f"{int((same & decided).sum())}/{int(decided.sum())}",
            "search_near_ties": int(tie.sum()), "search_mismatch": int((~same & ~tie).sum())}


def verify(pipe, scene, P, fr, nthreads=0, seed=0):
    """The device step against the FP64 oracle: per pass the whole integer-search grid, the
    bad-point removal, IC-GN from the device's initial guesses (flags, iteration counts,
    u/v and the warp gradients F); the triangulated XYZ of both frames."""
    import oracle as O

    n = pipe.n
    coords = pipe.coords_np
    coordsR = pipe.coordsR.t().cpu().numpy()
    passes = {"stereo": ("S", "L0", "R0", "gL0", coords, P["tol_stereo"], P["s_stereo"]),
              "left": ("L", "L0", "L1", "gL0", coords, P["tol_temp"], P["s_temp"]),
              "right": ("R", "R0", "R1", "gR0", coordsR, P["tol_temp"], P["s_temp"])}
    res = {}
    nx, ny = pipe.nx, pipe.ny
    gi = np.arange(nx * ny)
    ii = (1 + (gi % nx) * P["step"]).astype(np.int32)
    jj = (1 + (gi // nx) * P["step"]).astype(np.int32)
    for name, (k, fk, gk, gradk, crd, tol, s) in passes.items():
        b = pipe.buf[k]
        U0 = b["U0"].cpu().numpy()
        U = b["U"].cpu().numpy()
        F = b["F"].cpu().numpy()
        conv = b["conv"].cpu().numpy()
        frame = O.Frame(fr[fk], fr[gk], None, fr[gradk][0], fr[gradk][1])
        t0 = time.perf_counter()
        ref = O.local_icgn(frame, crd, U0, P["w"], tol, variant=1, nthreads=nthreads)
        t_icgn = time.perf_counter() - t0
        fg = (conv > 0) & (conv < 100)
        fo = (ref["conv"] > 0) & (ref["conv"] < 100)
        d = np.abs(U - ref["U"]).reshape(-1, 2)
        dF = np.abs(F - ref["F"]).reshape(-1, 4)
        ok = fg & fo & np.all(d <= 0.01, axis=1)
        both = fg & fo
        # integer search over the whole grid (same clamps as the device run); the device's
        # nY x nX column-major grids as [j][i] arrays, flattened x fastest (the ii, jj order)
        gu2 = b["u"].cpu().numpy().reshape(nx, ny).T
        gv2 = b["v"].cpu().numpy().reshape(nx, ny).T
        gu, gv = gu2.ravel(), gv2.ravel()
        t0 = time.perf_counter()
        sref = O.search_check(fr[fk], fr[gk], [s, s], P["size"], P["size"], ii, jj, P["w"], nthreads=nthreads)
        t_search = time.perf_counter() - t0
        sp = search_parity(gu, gv, sref)
        # the bad-point removal over the whole grid against the oracle's, from the same search
        uo, vo, bad = O.remove_outliers(gu2, gv2, 100.0)
        du = b["uo"].cpu().numpy().reshape(nx, ny).T
        dv = b["vo"].cpu().numpy().reshape(nx, ny).T
        nan_same = np.array_equal(np.isnan(du), np.isnan(uo)) and np.array_equal(np.isnan(dv), np.isnan(vo))
        out_err = float(max(np.nanmax(np.abs(du - uo)), np.nanmax(np.abs(dv - vo)))) if nan_same else None
        res[name] = {"n": int(n), "converged_gpu": int(fg.sum()), "converged_oracle": int(fo.sum()),
                     "counted": int(ok.sum()), "flag_match": float(np.mean(fg == fo)),
                     "iterations_match": float(np.mean(conv == ref["conv"])),
                     "uv_max_err": float(d[both].max()) if both.any() else None,
                     "F_max_err": float(dF[both].max()) if both.any() else None,
                     **sp, "outliers_removed": int(bad.size), "outliers_max_err": out_err,
                     "oracle_icgn_s": t_icgn, "oracle_search_s": t_search}
    # FP64 triangulation of both frames' matched pairs against the oracle's DLT
    tri = {}
    for kf in range(2):
        pairs = pipe.pairs[kf].cpu().numpy().T
        xyz = pipe.xyz[kf]["xyz"].cpu().numpy().reshape((n, 3), order="F")
        xo, _ = O.triangulate(pairs, scene.KL, scene.KR, scene.R_rl, scene.T_rl)
        fin = np.all(np.isfinite(xo), axis=1)
        same_nan = bool(np.array_equal(fin, np.all(np.isfinite(xyz), axis=1)))
        rel = np.linalg.norm(xyz[fin] - xo[fin], axis=1) / np.linalg.norm(xo[fin], axis=1)
        tri[f"frame{kf}"] = {"points": int(fin.sum()), "nan_rows_match": same_nan,
                             "xyz_rel_err": float(rel.max()) if rel.size else None}
    res["triangulation"] = tri
    return res


# ----------------------------------------------------------------------------------
# CPU (oracle) path on a bounded sample: baseline and reference arm
# ----------------------------------------------------------------------------------
def cpu_sample(scene, P, per_pass, nthreads, seed=0):
    """Time the FP64 CPU restatement of the same workload on `per_pass` subsets per pass:
    normalise/gradient (scaled to the sample), integer search and IC-GN."""
    import oracle as O

    M = N = P["size"]
    w, st = P["w"], P["step"]
    coords, nx, ny = grid_coords(M, N, w, st)
    n = coords.shape[0]
    t0 = time.perf_counter()
    fr = oracle_frames(scene, P)
    t_prep_full = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    total_t = 0.0
    conv_count = 0
    done = 0
    for name, (fk, gk, gradk, s, tol) in {"stereo": ("L0", "R0", "gL0", P["s_stereo"], P["tol_stereo"]),
                                           "left": ("L0", "L1", "gL0", P["s_temp"], P["tol_temp"]),
                                           "right": ("R0", "R1", "gR0", P["s_temp"], P["tol_temp"])}.items():
        pick = rng.choice(nx * ny, size=per_pass, replace=False)
        t1 = time.perf_counter()
        ii = 1 + (pick % nx) * st
        jj = 1 + (pick // nx) * st
        sub = O.search_list(fr[fk], fr[gk], [s, s], M, N, ii, jj, w, nthreads=nthreads)
        U0 = np.nan_to_num(sub[:, :2]).ravel()
        crd = np.stack([ii + w / 2.0, jj + w / 2.0], 1).astype(np.float64)
        frame = O.Frame(fr[fk], fr[gk], None, fr[gradk][0], fr[gradk][1])
        r = O.local_icgn(frame, crd, U0, w, tol, variant=1, nthreads=nthreads)
        total_t += time.perf_counter() - t1
        conv_count += int(np.sum((r["conv"] > 0) & (r["conv"] < 100)))
        done += per_pass
    total_t += t_prep_full * done / (3 * n)
    return conv_count / total_t, total_t, done, conv_count


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args, P):
    """--impl reference: the CPU restatement (FP64 oracle) of the reference path, all host
    threads, each step a bounded sample of the workload."""
    import oracle as O

    O.build()
    scene = make_scene(args.workload, args.seed)
    nthr = host_threads()
    per = args.ref_per_pass
    cpu_sample(scene, P, max(2, per // 4), nthr, seed=99)  # warm-up (page-in, thread pool)
    vals, times, conv_tot, done_tot = [], [], 0, 0
    for k in range(args.steps):
        v, t, done, conv = cpu_sample(scene, P, per, nthr, seed=k)
        vals.append(v)
        times.append(t)
        conv_tot += conv
        done_tot += done
    value = conv_tot / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded analytic speckle rendering)",
            "config": {"workload": args.workload, **P},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthr, "kind": "port",
                             "sample": f"{per} subsets per pass x 3 passes per step (search + IC-GN), "
                                       f"prep scaled to the sample; FP64 C++ restatement, OpenMP"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------
# learned vs FFT initial guess (learned2048)
# ----------------------------------------------------------------------------------
LEARNED_METRIC = "converged IC-GN subsets/s at <=0.01 px vs FP64 oracle; learned vs FFT init, 1 B200"


class LearnedBench:
    """The two initial-guess paths on one device, each a pass over one frame pair (uint8
    2048 x 2048, resident): load + normalise + gradients, then
      learned: network prediction -> IC-GN from [F0 U0] (its last iteration gives the ZNCC
               check) -> integer search + IC-GN on the failed subsets (the fallback);
      fft:     whole-field integer search -> outlier removal -> Init (inpaint) -> IC-GN from
               [0 U0] (LocalICGN's reference path).
    Both on the same integer-search grid (ROI [roi+1, size-roi], winsize w, step), all work on
    one stream.  The learned path's timed frames go through a LearnedPipeline over two
    contexts (frame k queued before the host reads frame k-1's fallback count)."""

    def __init__(self, A, torch, P, device, autotune=True):
        from aldic_b200 import learned as L
        from aldic_b200 import train_net

        self.A, self.T, self.P = A, torch, P
        M = N = P["size"]
        self.M, self.N = M, N
        self.gx, self.gy = [P["roi"] + 1, M - P["roi"]], [P["roi"] + 1, N - P["roi"]]
        di = device.index or 0
        nodes = L.search_nodes(self.gx, self.gy, P["w"], P["step"])[0].shape[1]
        self.net = L.ProposalNet(di, max_batch=min(16384, (nodes + 7) // 8 * 8))
        self.net.set_params(np.load(train_net.DEFAULT_WEIGHTS))
        self.ctx = A.Context(di)
        self.ctx2 = A.Context(di)  # the learned path's second frame in flight
        for c in (self.ctx, self.ctx2):
            c.set_option(A.OPT_AUTOTUNE, 1 if autotune else 0)
        self.pipe = L.LearnedPipeline(self.net, [self.ctx, self.ctx2], P["search"], self.gx, self.gy, P["w"],
                                      P["step"], P["tol"])
        self.li = self.pipe.lis[0]
        self.stream = self.li.stream
        self.n, self.nx, self.ny = self.li.n, self.li.nx, self.li.ny
        f64 = dict(dtype=torch.float64, device=device)
        g, n = self.nx * self.ny, self.n
        self.fb = {k: torch.empty(g, **f64) for k in ("x", "y", "u", "v", "phi")}
        self.fb.update({"U0": torch.empty(2 * n, **f64), "U": torch.empty(2 * n, **f64),
                        "F": torch.empty(4 * n, **f64), "conv": torch.empty(n, dtype=torch.int32, device=device)})
        self.fft_icgn_events = None

    def load(self, ref, deff, ctx=None):
        c = ctx if ctx is not None else self.ctx
        c.load_image_raw(0, ref, self.gx, self.gy, want_stats=False, shape=(self.M, self.N))
        c.load_image_raw(1, deff, self.gx, self.gy, want_stats=False, shape=(self.M, self.N))
        c.compute_gradients()

    def learned(self, ref, deff):
        """One frame, finished before the call returns (the first context)."""
        with self.T.cuda.stream(self.stream):
            self.load(ref, deff)
        return self.li.run()

    def learned_pipelined(self, ref, deff):
        """One frame pushed through the two-context pipeline; returns the previous frame's
        fallback count (None for the first)."""
        done = self.pipe.push(lambda ctx: self.load(ref, deff, ctx))
        return None if done is None else done.n_fallback

    def learned_flush(self):
        done = self.pipe.flush()
        return None if done is None else done.n_fallback

    def fft(self, ref, deff):
        P, c, b = self.P, self.ctx, self.fb
        with self.T.cuda.stream(self.stream):
            self.load(ref, deff)
            c.integer_search([P["search"]] * 2, self.gx, self.gy, P["w"], P["step"], out=b)
            u, v = b["u"].view(self.nx, self.ny), b["v"].view(self.nx, self.ny)
            c.remove_outliers(u, v, 100.0)
            c.init_u0(u, v, out=b["U0"])
            self.li._timed(self.fft_icgn_events, lambda: c.local_icgn(
                self.A.QUADTREE, self.li.coords, b["U0"], P["w"], P["tol"], want_H=False, want_mark=False, out=b))

    def snapshot(self, which):
        """Host copies of the last pass's results (waits for the stream)."""
        self.stream.synchronize()
        b = self.li.buf if which == "learned" else self.fb
        keys = ("U0", "F0", "U", "F", "conv", "fallback") if which == "learned" else ("U0", "U", "F", "conv")
        return {k: b[k].cpu().numpy() for k in keys}

    def launches(self):
        return self.ctx.launches + self.ctx2.launches + self.net.launches

    def close(self):
        self.net.close()
        self.ctx.close()
        self.ctx2.close()


def learned_frames(P, seeds, device):
    from aldic_b200 import synth_gpu

    return [synth_gpu.field_pair(s, P["size"], P["size"], umax=P["umax"], gmax=P["gmax"], device=device)
            for s in seeds]


def learned_verify(bench, pair, res_l, res_f, nthreads):
    """Both paths' results on one frame against the FP64 oracle run from the same initial
    guesses (the learned path's [F0 U0], the search's fallback guesses included; the FFT
    path's [0 U0]) on the same normalised frames."""
    import oracle as O

    M, N = bench.M, bench.N
    P = bench.P
    ref = pair.ref.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    deff = pair.deff.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    f, _ = O.normalize(ref, bench.gx, bench.gy)
    g, _ = O.normalize(deff, bench.gx, bench.gy)
    gx, gy = O.gradient(f)
    frame = O.Frame(f, g, None, gx, gy)
    crd = bench.li.coords.cpu().numpy().T.copy()
    out = {}
    for name, r in (("learned", res_l), ("fft", res_f)):
        F0 = r["F0"] if name == "learned" else None
        t0 = time.perf_counter()
        o = O.local_icgn(frame, crd, r["U0"], P["w"], P["tol"], variant=1, nthreads=nthreads, F0=F0)
        t_o = time.perf_counter() - t0
        fg = (r["conv"] > 0) & (r["conv"] < 100)
        fo = (o["conv"] > 0) & (o["conv"] < 100)
        d = np.abs(r["U"] - o["U"]).reshape(-1, 2)
        dF = np.abs(r["F"] - o["F"]).reshape(-1, 4)
        ok = fg & fo & np.all(d <= 0.01, axis=1)
        both = fg & fo
        out[name] = {"n": int(fg.size), "converged_gpu": int(fg.sum()), "converged_oracle": int(fo.sum()),
                     "counted": int(ok.sum()), "flag_match": float(np.mean(fg == fo)),
                     "iterations_match": float(np.mean(r["conv"] == o["conv"])),
                     "mean_iterations": float(r["conv"][fg].mean()) if fg.any() else None,
                     "uv_max_err": float(d[both].max()) if both.any() else None,
                     "F_max_err": float(dF[both].max()) if both.any() else None, "oracle_s": t_o}
    # the network's guesses against the converged solutions (non-fallback subsets)
    keep = ~res_l["fallback"] & (res_l["conv"] > 0) & (res_l["conv"] < 100)
    du = np.hypot(*(res_l["U0"] - res_l["U"]).reshape(-1, 2)[keep].T)
    dF0 = np.abs(res_l["F0"] - res_l["F"]).reshape(-1, 4)[keep]
    okf = (res_f["conv"] > 0) & (res_f["conv"] < 100)
    dus = np.hypot(*(res_f["U0"] - res_f["U"]).reshape(-1, 2)[okf].T)
    both = keep & okf
    out["guess"] = {"net_u_err_px_p50": float(np.median(du)), "net_u_err_px_p99": float(np.percentile(du, 99)),
                    "net_F_err_p50": float(np.median(dF0)),
                    "zero_F_err_p50": float(np.median(np.abs(res_l["F"].reshape(-1, 4)[keep]))),
                    "search_u_err_px_p50": float(np.median(dus)),
                    "learned_vs_fft_uv_max": float(np.abs(res_l["U"] - res_f["U"]).reshape(-1, 2)[both].max())
                    if both.any() else None,
                    "fallback": int(res_l["fallback"].sum())}
    return out


def net_flops(M, N, n):
    """Algorithmic FLOPs of one prediction: conv1 (9 taps x 32) and conv2 (288 x 32) over the
    two whole images' output pixels, then per subset the 64 x 81 correlation entries (32
    channels), conv3 (16 x 64 x 729), conv4 (16 x 64 x 576), FC1 (1024 x 128), FC2 (128 x 6);
    2 per multiply-add."""
    M1, N1 = (M + 1) // 2, (N + 1) // 2
    M2, N2 = (M1 + 1) // 2, (N1 + 1) // 2
    per_image = M1 * N1 * 32 * 9 + M2 * N2 * 32 * 288
    per_subset = 64 * 81 * 32 + 16 * 64 * 729 + 16 * 64 * 576 + 1024 * 128 + 128 * 6
    return 2.0 * (2 * per_image + n * per_subset)


def learned_cpu_sample(P, pair, gx, gy, per, nthreads, seed=0):
    """The FP64 CPU restatement of the reference's path on this workload (integer search +
    IC-GN from [0 U0], LocalICGN), timed on `per` grid subsets of one frame, the frame's
    normalisation and gradients scaled to the sample."""
    import oracle as O

    M = N = P["size"]
    w, st, s = P["w"], P["step"], P["search"]
    ref = pair.ref.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    deff = pair.deff.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    t0 = time.perf_counter()
    f, _ = O.normalize(ref, gx, gy)
    g, _ = O.normalize(deff, gx, gy)
    dfx, dfy = O.gradient(f)
    t_prep = time.perf_counter() - t0
    nx, ny = O.search_grid(gx, gy, w, st)
    rng = np.random.default_rng(seed)
    pick = rng.choice(nx * ny, size=min(per, nx * ny), replace=False)
    ii = gx[0] + (pick % nx) * st
    jj = gy[0] + (pick // nx) * st
    t1 = time.perf_counter()
    sub = O.search_list(f, g, [s, s], gx[1], gy[1], ii, jj, w, nthreads=nthreads)
    U0 = np.nan_to_num(sub[:, :2]).ravel()
    crd = np.stack([ii + w / 2.0, jj + w / 2.0], 1).astype(np.float64)
    r = O.local_icgn(O.Frame(f, g, None, dfx, dfy), crd, U0, w, P["tol"], variant=1, nthreads=nthreads)
    t = time.perf_counter() - t1 + t_prep * pick.size / (nx * ny)
    conv = int(np.sum((r["conv"] > 0) & (r["conv"] < 100)))
    return conv / t, t, int(pick.size), conv


def run_learned(args, P):
    import torch

    import aldic_b200 as A
    from aldic_b200 import train_net

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    # weak scaling: every rank its own held-out frames, no data-path collective
    F = P["frames"]
    base = 50000 + 1000 * (args.seed + rank)
    pairs = learned_frames(P, [base + k for k in range(F)], dev)
    warm = learned_frames(P, [base + 900 + k for k in range(max(args.warmup, 3))], dev)
    bench = LearnedBench(A, torch, P, dev, autotune=not args.no_autotune)
    st = bench.stream
    for p in warm:  # warm-up: the autotuner's first calls (both contexts), page-in
        bench.fft(p.ref, p.deff)
        bench.learned_pipelined(p.ref, p.deff)
    bench.learned_flush()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()

    def timed(fn, finish=None):
        clocks = ClockSampler(local_rank)
        l0 = bench.launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        ev0.record(st)
        extra = [fn(pairs[k % F].ref, pairs[k % F].deff) for k in range(args.steps)]
        if finish is not None:
            extra.append(finish())
        ev1.record(st)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1), clocks.stop(), bench.launches() - l0, extra

    # the learned path: frames pipelined over two contexts (the host's wait for a frame's
    # fallback count overlaps the device's work on the next frame)
    pred_ev, icgn_ev = [], []
    for li in bench.pipe.lis:
        li.predict_events, li.icgn_events = pred_ev, icgn_ev
    ms_l, clk_l, launches_l, fallbacks = timed(bench.learned_pipelined, bench.learned_flush)
    fallbacks = [f for f in fallbacks if f is not None]
    for li in bench.pipe.lis:
        li.predict_events = li.icgn_events = None
    if dist:
        dist.barrier()
    bench.fft_icgn_events = []
    ms_f, clk_f, launches_f, _ = timed(bench.fft)
    fft_icgn_ev, bench.fft_icgn_events = bench.fft_icgn_events, None
    predict_ms = float(np.mean([a.elapsed_time(b) for a, b in pred_ev]))
    icgn_ms = float(np.mean([a.elapsed_time(b) for a, b in icgn_ev]))
    fft_icgn_ms = float(np.mean([a.elapsed_time(b) for a, b in fft_icgn_ev]))

    # per frame: both paths' results (deterministic: the timed passes produced the same) and
    # their verification against the FP64 oracle
    import oracle as O

    O.build()
    nthr = host_threads()
    counted_l, counted_f, ver, conv_frames = [], [], [], []
    for k, p in enumerate(pairs[:min(F, args.steps)]):
        bench.learned(p.ref, p.deff)
        rl = bench.snapshot("learned")
        conv_frames.append(rl["conv"])
        bench.fft(p.ref, p.deff)
        rf = bench.snapshot("fft")
        v = learned_verify(bench, p, rl, rf, nthr) if not args.no_verify else None
        ver.append(v)
        counted_l.append(v["learned"]["counted"] if v else int(((rl["conv"] > 0) & (rl["conv"] < 100)).sum()))
        counted_f.append(v["fft"]["counted"] if v else int(((rf["conv"] > 0) & (rf["conv"] < 100)).sum()))
    nF = len(counted_l)
    tot_l = float(sum(counted_l[k % nF] for k in range(args.steps)))
    tot_f = float(sum(counted_f[k % nF] for k in range(args.steps)))
    # end to end through the public API: frames from pinned host memory, results back to it
    e2e_steps = max(1, args.e2e_steps)
    M, N, n = bench.M, bench.N, bench.n
    host = []
    for p in pairs[:min(nF, e2e_steps)]:
        hr = torch.empty(M * N, dtype=torch.uint8, pin_memory=True)
        hd = torch.empty(M * N, dtype=torch.uint8, pin_memory=True)
        hr.copy_(p.ref)
        hd.copy_(p.deff)
        host.append((hr.numpy().reshape((M, N), order="F"), hd.numpy().reshape((M, N), order="F")))
    hU = torch.empty(2 * n, dtype=torch.float64, pin_memory=True)
    hc = torch.empty(n, dtype=torch.int32, pin_memory=True)
    for k in range(2):  # untimed: both contexts stage host frames once (their staging buffers grow)
        hr, hd = host[k % len(host)]
        bench.pipe.push(lambda ctx, hr=hr, hd=hd: bench.load(hr, hd, ctx))
    bench.pipe.flush()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    def fetch(done):  # a finished frame's U and codes to pinned host memory, on the stream
        if done is not None:
            with torch.cuda.stream(st):
                hU.copy_(done.buf["U"], non_blocking=True)
                hc.copy_(done.buf["conv"], non_blocking=True)

    for k in range(e2e_steps):
        hr, hd = host[k % len(host)]
        fetch(bench.pipe.push(lambda ctx, hr=hr, hd=hd: bench.load(hr, hd, ctx)))
    fetch(bench.pipe.flush())
    e1.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_conv = float(np.mean([counted_l[k % len(host)] for k in range(e2e_steps)]))
    h2d, d2h = 2 * M * N, hU.numel() * 8 + hc.numel() * 4

    if dist:
        t = torch.tensor([ms_l, ms_f, e2e_ms], dtype=torch.float64, device=dev)
        tot = torch.tensor([tot_l, tot_f, e2e_conv], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        ms_l, ms_f, e2e_ms = float(t[0]), float(t[1]), float(t[2])
        tot_l, tot_f, e2e_conv = float(tot[0]), float(tot[1]), float(tot[2])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, tcpu, done, conv = learned_cpu_sample(P, pairs[0], bench.gx, bench.gy, args.cpu_per_pass, nthr)
        cpu = {"value": v, "unit": UNIT, "cores": nthr, "kind": "port",
               "sample": f"{done} grid subsets of one 2048 x 2048 frame: integer search + IC-GN from [0 U0] "
                         f"(the reference's path; it has no learned guess), normalisation and gradients scaled "
                         f"to the sample; {tcpu:.1f} s of CPU wall time, FP64 C++ restatement, OpenMP"}

    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        fp32_peak = measure_fp32_peak(torch, dev)
        icgn_work = float(np.mean([icgn_flops(c, P["w"]) for c in conv_frames])) if conv_frames else None
        nf = net_flops(M, N, n)
        bf16_peak = peaks.get("bf16_tflops")
        summary = {}
        try:
            summary = json.load(open(os.path.splitext(train_net.DEFAULT_WEIGHTS)[0] + ".json"))
        except Exception:
            pass

        def agg(key):
            vs = [v[key] for v in ver if v]
            if not vs:
                return None
            return {"counted": int(sum(x["counted"] for x in vs)), "n": int(sum(x["n"] for x in vs)),
                    "converged_gpu": int(sum(x["converged_gpu"] for x in vs)),
                    "flag_match_min": min(x["flag_match"] for x in vs),
                    "iterations_match_min": min(x["iterations_match"] for x in vs),
                    "mean_iterations": float(np.mean([x["mean_iterations"] for x in vs])),
                    "uv_max_err": max(x["uv_max_err"] for x in vs), "F_max_err": max(x["F_max_err"] for x in vs)}

        guess = None
        if ver and ver[0]:
            gk = ver[0]["guess"].keys()
            guess = {k: (float(np.mean([v["guess"][k] for v in ver])) if k != "fallback"
                         else int(sum(v["guess"][k] for v in ver))) for k in gk}
        value, fft_value = tot_l / (ms_l * 1e-3), tot_f / (ms_f * 1e-3)
        line = {
            "metric": LEARNED_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_l / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (BF16 network, FP64 solve and re-decisions)",
            "data": "synthetic (seeded analytic speckle rendering; held-out frames, not in the training set)",
            "config": {"workload": args.workload, "subsets_per_frame": n, "frames_cycled": nF, **P,
                       "l2_flush": "each step a different frame; a step's working set (two 16 MiB FP32 images "
                                   "and gradients, 2 x 16 MiB feature maps, 356 MiB of conv3 input rows) "
                                   "exceeds the 126 MB L2"},
            "fft_init": {"value": fft_value, "unit": UNIT, "ms_per_step": ms_f / args.steps,
                         "gpu_launches": int(launches_f), "clocks": clk_f},
            "learned_over_fft": value / fft_value,
            "gpu_launches": int(launches_l),
            "stage_ms": {"predict": predict_ms, "icgn_from_net_guess": icgn_ms, "icgn_from_search_guess": fft_icgn_ms},
            "fallback_rate": float(sum(fallbacks)) / (args.steps * n),
            "roofline": {"bound": "fp32", "kernel": "IC-GN call from the network's guess (classify, one-warp pass, "
                                                 "slow-subset pass, general and FP64 re-solve kernels)",
                         "achieved": icgn_work / (icgn_ms * 1e-3) / 1e12 if icgn_work else None,
                         "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": icgn_work / (icgn_ms * 1e-3) / 1e12 / fp32_peak if icgn_work and fp32_peak else None,
                         "traffic": None, "algorithmic_flops_per_call": icgn_work, "call_ms": icgn_ms,
                         "calls_timed": len(icgn_ev),
                         "flops_counted": "92 (w+1)^2 per subset-iteration + 50 (w+1)^2 per subset solved",
                         "peak_source": "measured on this GPU: the faster of a scalar FFMA and a packed FFMA2 loop"},
            "roofline_net": {"bound": "tensor", "kernel": "network prediction (whole-image conv1/conv2, tcgen05 "
                                                          "correlation, conv3/conv4/FC GEMMs)",
                             "achieved": nf / (predict_ms * 1e-3) / 1e12, "peak": bf16_peak, "unit": "TFLOP/s",
                             "frac": nf / (predict_ms * 1e-3) / 1e12 / bf16_peak if bf16_peak else None,
                             "algorithmic_flops_per_call": nf, "call_ms": predict_ms,
                             "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS burst)"},
            "network": {k: summary.get(k) for k in ("samples", "steps", "batch", "train_s", "data_s", "held_out")},
            "tuning": bench.ctx.tuning_report(),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_conv / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "clocks": clk_l,
            "verification": {"frames": nF, "learned": agg("learned"), "fft": agg("fft"), "guess": guess},
            "hbm_peak_gbs": peaks.get("hbm_gbs"),
        }
    bench.close()
    del pairs, warm
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_stereo:
            # the 1-GPU line also carries the stereo + temporal + triangulation step (its own
            # frames, timing and whole-grid oracle verification), run after the learned one
            sargs = argparse.Namespace(**vars(args))
            sargs.workload, sargs.no_cpu = "stereo2048", True
            try:
                sl = run_stereo(sargs, workload_params("stereo2048"), emit=False)
                line["stereo2048"] = {k: sl.get(k) for k in ("value", "unit", "ms_per_step", "gpu_launches", "config",
                                                             "roofline", "roofline_icgn", "e2e", "clocks",
                                                             "verification", "fp64_resolves")}
            except Exception as e:  # recorded, not fatal to the headline line
                line["stereo2048"] = {"error": f"{type(e).__name__}: {e}"}
        print(json.dumps(line), flush=True)


def run_reference_learned(args, P):
    """--impl reference on learned2048: the reference's own path for it (integer search +
    IC-GN from [0 U0]; it has no learned guess) in the FP64 CPU restatement, all host threads,
    each step a bounded sample of one held-out frame's grid subsets."""
    import oracle as O

    O.build()
    try:
        import torch

        device = "cuda" if torch.cuda.is_available() else "cpu"
    except Exception:
        device = "cpu"
    nthr = host_threads()
    frames = learned_frames(P, [50000 + 1000 * args.seed + k for k in range(min(args.steps, P["frames"]))], device)
    M = P["size"]
    gx = [P["roi"] + 1, M - P["roi"]]
    per = 3 * args.ref_per_pass
    learned_cpu_sample(P, frames[0], gx, gx, max(8, per // 8), nthr, seed=99)  # warm-up
    times, conv_tot = [], 0
    for k in range(args.steps):
        _, t, _, conv = learned_cpu_sample(P, frames[k % len(frames)], gx, gx, per, nthr, seed=k)
        times.append(t)
        conv_tot += conv
    value = conv_tot / sum(times)
    line = {"impl": "reference", "metric": LEARNED_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded analytic speckle rendering; held-out frames)",
            "config": {"workload": args.workload, **P},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthr, "kind": "port",
                             "sample": f"{per} grid subsets per step: integer search + IC-GN from [0 U0] (the "
                                       f"reference's path), normalisation and gradients scaled to the sample; "
                                       f"FP64 C++ restatement, OpenMP"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------
def run_stereo(args, P, emit=True):
    """The stereo2048 / stereo1024 step (see the module docstring); rank 0 returns its JSON
    line (and prints it when emit)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    import aldic_b200 as A

    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    # weak scaling: every rank owns its own seeded frame set; no data-path collective
    scene = make_scene(args.workload, args.seed + rank)
    pipe = StereoPipeline(A, torch, scene, P, dev, autotune=not args.no_autotune)
    stream = pipe.stream
    for _ in range(max(args.warmup, 3)):
        pipe.step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    l0 = pipe.launches()
    # dominant kernel: the correlation kernel of the stereo integer search, timed inside the
    # timed region by CUDA events the library records around that launch on the same stream
    cS = pipe.ctx["S"]
    cS.set_profiling(True)
    cS.profile_read()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pipe.icgn_events = []
    ev0.record(stream)
    for _ in range(args.steps):
        pipe.step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    ms_total = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = (pipe.launches() - l0)
    ms_step = ms_total / args.steps
    prof_ms, prof_n = cS.profile_read()
    cS.set_profiling(False)
    icgn_ms = float(np.mean([a.elapsed_time(b) for a, b in pipe.icgn_events]))
    pipe.icgn_events = None
    icgn_work = icgn_flops(pipe.buf["S"]["conv"].cpu().numpy(), P["w"])
    search_ms = prof_ms / max(prof_n, 1)
    flops = tile_flops(P["size"], P["size"], P["w"], P["step"], P["s_stereo"], P["s_stereo"])
    direct_flops = crop_flops(P["size"], P["size"], P["w"], P["step"], P["s_stereo"], P["s_stereo"])
    fp32_peak = measure_fp32_peak(torch, dev)

    # verification against the FP64 oracle (outside the timed region)
    if args.no_verify:
        ver = None
        counted = 3 * pipe.n
    else:
        import oracle as O

        O.build()
        fr = oracle_frames(scene, P)
        ver = verify(pipe, scene, P, fr, nthreads=host_threads())
        counted = sum(v["counted"] for k, v in ver.items() if k != "triangulation")

    # end to end through the public API with host buffers
    e2e = e2e_measure(A, scene, P, args.e2e_steps, local_rank) if args.e2e_steps > 0 else \
        {"ms": float("nan"), "converged": 0.0, "h2d": 0, "d2h": 0}

    if dist:
        t = torch.tensor([ms_step, -float(counted), e2e["ms"], search_ms], dtype=torch.float64, device=dev)
        tot = torch.tensor([float(counted), e2e["converged"]], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        ms_step_all, e2e_ms_all = float(t[0]), float(t[2])
        counted_all, e2e_conv_all = float(tot[0]), float(tot[1])
    else:
        ms_step_all, e2e_ms_all, counted_all, e2e_conv_all = ms_step, e2e["ms"], float(counted), e2e["converged"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthr = host_threads()
        v, tcpu, done, conv = cpu_sample(scene, P, args.cpu_per_pass, nthr)
        cpu = {"value": v, "unit": UNIT, "cores": nthr, "kind": "port",
               "sample": f"{args.cpu_per_pass} subsets per pass x 3 passes (integer search + IC-GN), prep scaled; "
                         f"{tcpu:.1f} s of CPU wall time"}

    if rank == 0:
        import json as _json

        peaks = {}
        try:
            peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        achieved = flops / (search_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": counted_all / (ms_step_all * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step_all, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 solve/fit/triangulation)",
            "data": "synthetic (seeded analytic speckle rendering)",
            "config": {"workload": args.workload, "subsets_per_pass": pipe.n, "passes": 3,
                       "l2_flush": "inputs (4 x 8 MiB frames + 3 contexts of FP32 images/gradients/integral images) "
                                   "exceed the 126 MB L2 across a step", **P},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "kernel": "ncc_tile_kernel (stereo integer search, shared products)",
                         "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak if fp32_peak else None,
                         "traffic": TILE_TRAFFIC.get(args.workload), "traffic_unit": "bytes per launch",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel "
                                           "at this workload (separate capture)",
                         "peak_source": "measured on this GPU: the faster of a scalar FFMA and a packed FFMA2 "
                                        "loop (MEASURED_PEAKS.json holds only HBM and bf16 tensor peaks)",
                         "algorithmic_flops_per_launch": flops, "flops_counted": "products only (2 per f*g)",
                         "direct_correlation_flops": direct_flops, "launch_ms": search_ms,
                         "launches_timed": prof_n},
            "roofline_icgn": {"bound": "fp32", "kernel": "stereo IC-GN call (classify, one-warp pass, slow-subset "
                                                      "pass, general and FP64 re-solve kernels)",
                              "achieved": icgn_work / (icgn_ms * 1e-3) / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
                              "frac": icgn_work / (icgn_ms * 1e-3) / 1e12 / fp32_peak if fp32_peak else None,
                              "algorithmic_flops_per_call": icgn_work, "call_ms": icgn_ms,
                              "calls_timed": args.steps,
                              "flops_counted": "92 (w+1)^2 per subset-iteration (iterations = the codes; 100 for "
                                               "code 101) + 50 (w+1)^2 per subset solved",
                              "peak_source": "the measured FP32 peak above"},
            "tuning": pipe.tuning(),
            "fp64_resolves": {k: c.get_option(A.STAT_FP64_RESOLVES) for k, c in pipe.ctx.items()},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_conv_all / (e2e_ms_all * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
            "clocks": clk,
            "verification": ver,
            "hbm_peak_gbs": peaks.get("hbm_gbs"),
        }
        if emit:
            print(json.dumps(line), flush=True)
    pipe.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="learned2048",
                    choices=["learned2048", "learned1024", "stereo2048", "stereo1024", "temporal512", "quadtree2048",
                             "sequence4096"],
                    help="learned2048: learned vs FFT initial guess on held-out 2048 x 2048 frames (the "
                         "headline); stereo2048: the stereo + temporal + triangulation step; temporal512 and "
                         "quadtree2048: the 2D and quadtree/Subpb1 configurations; sequence4096: the 50-frame "
                         "4096 x 3000 stereo sequence with per-frame latency (separate JSON lines)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ref-per-pass", type=int, default=200)
    ap.add_argument("--cpu-per-pass", type=int, default=1200)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="the library's default configurations instead of the autotuner's (profiling runs: timings "
                         "under a profiler would mislead the tuner)")
    ap.add_argument("--no-stereo", action="store_true",
                    help="learned2048: skip the stereo2048 step that the 1-GPU line carries as a sub-object")
    args = ap.parse_args()
    P = workload_params(args.workload)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            if args.workload in ("learned2048", "learned1024"):
                run_reference_learned(args, P)
            elif args.workload in ("sequence4096", "temporal512", "quadtree2048"):
                print(json.dumps({"impl": "reference", "unavailable": f"{args.workload} times the FP64 CPU oracle "
                                  "on its own sample of the workload, from the device run's inputs (cpu_baseline "
                                  "of the ours line)"}), flush=True)
            else:
                run_reference(args, P)
        return
    if args.workload in ("learned2048", "learned1024"):
        run_learned(args, P)
        return
    if args.workload == "sequence4096":
        if rank == 0:
            run_sequence(args, P)
        return
    if args.workload in ("temporal512", "quadtree2048"):
        if rank == 0:
            run_aux(args, P)
        return

    run_stereo(args, P)


# ----------------------------------------------------------------------------------
# the 2D temporal (512^2) and quadtree ALDIC (2048^2, hole + notch, Subpb1) workloads
# ----------------------------------------------------------------------------------
def admm_beta(betas, errs):
    """The reference's beta for the first frame (aldic_b200.api.subpb2_beta)."""
    from aldic_b200.api import subpb2_beta

    return subpb2_beta(betas, errs)


def run_aux(args, P):
    """temporal512: LocalICGN on a 512^2 affine pair, FFT-search init.
    quadtree2048: one ALDIC frame on a 2048^2 plate with a hole and an edge notch:
    search, bad-point removal, Init, LocalICGNQuadtree on the quadtree mesh of
    GenerateQuadtreeMesh, the global step with the first frame's beta tuning, and two ADMM
    rounds of Subpb1Quadtree + Subpb2Quadtree.  Device-resident; verified on the oracle."""
    import torch

    import aldic_b200 as A
    from aldic_b200 import synth

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    T = torch
    f64 = dict(dtype=T.float64, device=dev)
    quad = args.workload == "quadtree2048"
    if quad:
        sc = synth.plate_with_hole(seed=args.seed, size=2048, hole_r=300.0, peak=5.0, sin_amp=0.5, sin_wl=200.0)
        mask = sc.mask
    else:
        sc = synth.temporal_affine(seed=args.seed)
        mask = None
    M, N = sc.ref.shape
    w, st = P["w"], P["step"]
    gx, gy = [1, M], [1, N]
    # search grid (XList rule) and the solve mesh
    gcoords, nx, ny = grid_coords(M, N, w, st)
    g = nx * ny
    if quad:
        # MeshSetUp on the search grid, refined at the mask's edges by GenerateQuadtreeMesh
        # (elements down to min_elem px): host set-up, as the reference builds its mesh once
        mesh0 = A.MeshSetUp(gcoords[:, 0].reshape(ny, nx), gcoords[:, 1].reshape(ny, nx),
                            {"winstepsize": st, "ImgSize": [M, N]})
        mesh0["elementMinSize"] = P["min_elem"]
        qmesh, _, _ = A.GenerateQuadtreeMesh(np.zeros(2 * g), None, mask, mesh0, {"winstepsize": st, "winsize": w})
        coords_np, E_np, dir_np = qmesh["coordinatesFEM"], qmesh["elementsFEM"], qmesh["dirichlet"]
        # the ADMM loop's uniform winsize_List
        wl_np = np.full(coords_np.shape[0], w, dtype=np.int32)
        wl = T.from_numpy(np.concatenate([wl_np, wl_np])).to(dev)  # n x 2 column-major (wx, wy)
        # U0 carried from the grid to the mesh nodes by bilinear weights (GenerateQuadtreeMesh
        # carries it by linear interpolation; the two agree on the grid's edges)
        fx = (coords_np[:, 0] - gcoords[0, 0]) / st
        fy = (coords_np[:, 1] - gcoords[0, 1]) / st
        i0 = np.clip(np.floor(fx), 0, nx - 2).astype(np.int64)
        j0 = np.clip(np.floor(fy), 0, ny - 2).astype(np.int64)
        tx, ty = fx - i0, fy - j0
        k00 = i0 + j0 * nx
        tr_idx = T.from_numpy(np.stack([k00, k00 + 1, k00 + nx, k00 + nx + 1])).to(dev)
        tr_w = T.from_numpy(np.stack([(1 - tx) * (1 - ty), tx * (1 - ty), (1 - tx) * ty, tx * ty])).to(dev)
        betas = [c * float(st) ** 2 * P["mu"] for c in (1e-3, 1e-2, 1e-1)]
    else:
        coords_np = gcoords
    n = coords_np.shape[0]
    coords = T.from_numpy(np.ascontiguousarray(coords_np.T)).to(dev)
    raw = {k: T.from_numpy(np.asfortranarray(img).ravel(order="F").copy()).to(dev) for k, img in
           (("ref", sc.ref), ("def", sc.deff))}
    mask_d = None if mask is None else T.from_numpy(np.asfortranarray(mask).ravel(order="F").copy()).to(dev)
    ctx = A.Context(0)
    stream = T.cuda.Stream(dev)
    ctx.set_stream(stream.cuda_stream)
    if quad:
        ctx.subpb2_set_mesh(n, E_np, dir_np)
    b = {"x": T.empty(g, **f64), "y": T.empty(g, **f64), "u": T.empty(g, **f64), "v": T.empty(g, **f64),
         "phi": T.empty(g, **f64), "U0": T.empty(2 * n, **f64), "U": T.empty(2 * n, **f64),
         "F": T.empty(4 * n, **f64), "H": T.empty(21 * n, **f64), "conv": T.empty(n, dtype=T.int32, device=dev),
         "mark": T.empty(n, dtype=T.uint8, device=dev), "Ug": T.empty(2 * g, **f64)}
    sub = [{"U": T.empty(2 * n, **f64), "conv": T.empty(n, dtype=T.int32, device=dev)} for _ in range(P.get("admm", 0))]
    cxy = coords.t()
    shp = (M, N)
    glob = {"U2": [T.empty(2 * n, **f64) for _ in range(3)], "out": T.empty(2 * n, **f64), "beta": None,
            "sub_in": None, "last": None}

    def aldic_frame():
        """ALDIC after the local step (func/TemporalMatch_quadtree_ST1.m:248-380): the global
        step with the first frame's beta tuning, then admm x (Subpb1, Subpb2, dual update),
        hole-edge nodes (markCoordHoleStrain) keeping the local result.  Bad local results
        take the initial guess (U) or 0 (F) where the reference fills them by
        natural-neighbour interpolation."""
        U1 = T.where(T.isnan(b["U"]), b["U0"], b["U"])
        F1 = T.nan_to_num(b["F"], nan=0.0)
        hole = b["mark"].bool().repeat_interleave(2)
        errs = []
        for k, bt in enumerate(betas):
            ctx.subpb2(coords, None, 2, bt, P["mu"], U1, F1, out=glob["U2"][k])
            errs.append(T.linalg.vector_norm(U1 - glob["U2"][k]))
        beta = admm_beta(betas, T.stack(errs).cpu().numpy())
        U2 = glob["U2"][2]
        if abs(beta - betas[2]) > np.finfo(float).eps:
            ctx.subpb2(coords, None, 2, beta, P["mu"], U1, F1, out=glob["out"])
            U2 = glob["out"]
        glob["beta"] = beta
        U2 = T.where(hole, U1, U2)
        vdual = U2 - U1
        for k in range(P["admm"]):
            if k == 0:
                glob["sub_in"] = (U2, vdual)
            ctx.subpb1(1, coords, U2, F1, vdual, P["mu"], P["tol_temp"], winsize=w, winsize_list=wl, out=sub[k])
            U1 = T.where(T.isnan(sub[k]["U"]), U2, sub[k]["U"])
            ctx.subpb2(coords, None, 2, beta, P["mu"], U1, F1, out=glob["out"])
            glob["last"] = (U1, F1, glob["out"].clone())
            U2 = T.where(hole, U1, glob["out"])
            vdual = U2 - U1

    def step():
        with T.cuda.stream(stream):
            ctx.load_image_raw(0, raw["ref"], gx, gy, want_stats=False, shape=shp)
            ctx.load_image_raw(1, raw["def"], gx, gy, want_stats=False, shape=shp)
            if quad:
                ctx.set_mask(mask_d)
            ctx.compute_gradients()
            ctx.integer_search([P["s_temp"]] * 2, gx, gy, w, st, out=b)
            # bad-point removal and Init over the search grid, then U0 on the mesh nodes
            ctx.remove_outliers(b["u"].view(nx, ny), b["v"].view(nx, ny), 100.0)
            ctx.init_u0(b["u"].view(nx, ny), b["v"].view(nx, ny), out=b["Ug"])
            if quad:
                b["U0"].view(n, 2).copy_((b["Ug"].view(-1, 2)[tr_idx] * tr_w[..., None]).sum(0))
            else:
                b["U0"].copy_(b["Ug"])
            ctx.local_icgn(1 if quad else 0, coords, b["U0"], w, P["tol_temp"], out=b)
            if quad:
                aldic_frame()

    for _ in range(max(args.warmup, 3)):
        step()
    T.cuda.synchronize(dev)
    clocks = ClockSampler(0)
    l0 = ctx.launches
    ev0, ev1 = T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    T.cuda.synchronize(dev)
    clk = clocks.stop()
    ms_step = ev0.elapsed_time(ev1) / args.steps
    launches = ctx.launches - l0
    solves = n * (1 + P.get("admm", 0))
    n_global = (3 + (abs(glob["beta"] - betas[2]) > np.finfo(float).eps) + P["admm"]) if quad else 0
    ver = None
    counted = None
    if not args.no_verify:
        import oracle as O

        O.build()
        f, _ = O.normalize(sc.ref.astype(np.float64), gx, gy)
        gimg, _ = O.normalize(sc.deff.astype(np.float64), gx, gy)
        gxo, gyo = O.gradient(f, mask)
        frame = O.Frame(f, gimg, mask, gxo, gyo)
        rng = np.random.default_rng(args.seed)
        pick = np.arange(n) if n <= 3000 else np.sort(rng.choice(n, 3000, replace=False))
        U0 = b["U0"].view(n, 2).cpu().numpy()[pick].ravel()
        U = b["U"].view(n, 2).cpu().numpy()[pick]
        conv = b["conv"].cpu().numpy()[pick]
        t0 = time.perf_counter()
        ref = O.local_icgn(frame, coords_np[pick], U0, w, P["tol_temp"], variant=1 if quad else 0,
                           nthreads=host_threads())
        t_icgn = time.perf_counter() - t0
        fg = (conv > 0) & (conv < 100)
        fo = (ref["conv"] > 0) & (ref["conv"] < 100)
        d = np.abs(U - ref["U"].reshape(-1, 2))
        ok = fg & fo & np.all(d <= 0.01, axis=1)
        ver = {"sample": int(len(pick)), "icgn_flag_match": float(np.mean(fg == fo)),
               "icgn_code_match": float(np.mean(conv == ref["conv"])),
               "icgn_uv_max_err": float(d[fg & fo].max()) if (fg & fo).any() else None,
               "icgn_counted_fraction": float(ok.mean()), "oracle_icgn_s": t_icgn}
        counted = ok.mean() * n
        if quad:
            # the first ADMM round's Subpb1 from the device's own inputs
            U2_in, vd_in = glob["sub_in"]
            Uin = U2_in.view(n, 2).cpu().numpy()[pick].ravel()
            vin = vd_in.view(n, 2).cpu().numpy()[pick].ravel()
            Fin = np.nan_to_num(b["F"].view(n, 4).cpu().numpy()[pick]).ravel()
            s1 = O.subpb1(frame, coords_np[pick], Uin, Fin, vin, P["mu"], P["tol_temp"],
                          winsize=w, winsize_list=np.stack([wl_np[pick], wl_np[pick]], 1), nthreads=host_threads())
            Us = sub[0]["U"].view(n, 2).cpu().numpy()[pick]
            cs = sub[0]["conv"].cpu().numpy()[pick]
            fgs = (cs > 0) & (cs < 100)
            fos = (s1["conv"] > 0) & (s1["conv"] < 100)
            ds = np.abs(Us - s1["U"].reshape(-1, 2))
            ver.update({"subpb1_flag_match": float(np.mean(fgs == fos)),
                        "subpb1_uv_max_err": float(ds[fgs & fos].max()) if (fgs & fos).any() else None})
            # the last global step, whole mesh, from the device's own inputs
            U1l, F1l, outl = (t.cpu().numpy() for t in glob["last"])
            t0 = time.perf_counter()
            ref2 = O.subpb2_quadtree(coords_np, E_np, 2, glob["beta"], P["mu"], U1l, F1l, dirichlet=dir_np)
            t_sp2 = time.perf_counter() - t0
            ver.update({"subpb2_max_err": float(np.abs(outl - ref2).max()),
                        "subpb2_field_max": float(np.abs(ref2).max()), "oracle_subpb2_s": t_sp2,
                        "beta": glob["beta"], "global_solves_per_step": int(n_global)})
    cpu = None
    if not args.no_cpu:
        import oracle as O

        O.build()
        f, _ = O.normalize(sc.ref.astype(np.float64), gx, gy)
        gimg, _ = O.normalize(sc.deff.astype(np.float64), gx, gy)
        gxo, gyo = O.gradient(f, mask)
        frame = O.Frame(f, gimg, mask, gxo, gyo)
        U0h = b["U0"].view(n, 2).cpu().numpy()
        Uh = np.nan_to_num(b["U"].view(n, 2).cpu().numpy())
        Fh = np.nan_to_num(b["F"].view(n, 4).cpu().numpy())
        rng = np.random.default_rng(args.seed + 7)
        cpu = {"kind": "port", "unit": "subsets/s" if not quad else "subset solves/s"}
        t_sp2_cpu = None
        for threads in (host_threads(), 1):
            ns = min(n, 900 if threads > 1 else 150)
            pk = np.sort(rng.choice(n, ns, replace=False))
            gpk = np.sort(rng.choice(nx * ny, min(nx * ny, 400 if threads > 1 else 60), replace=False))
            t0 = time.perf_counter()
            O.search_list(f, gimg, [P["s_temp"]] * 2, M, N, 1 + (gpk % nx) * st, 1 + (gpk // nx) * st, w,
                          nthreads=threads)
            t_search = (time.perf_counter() - t0) * (nx * ny) / len(gpk)
            t0 = time.perf_counter()
            O.local_icgn(frame, coords_np[pk], U0h[pk].ravel(), w, P["tol_temp"], variant=1 if quad else 0,
                         nthreads=threads)
            t_solve = time.perf_counter() - t0
            t_global = 0.0
            if quad:
                for _ in range(P["admm"]):
                    O.subpb1(frame, coords_np[pk], Uh[pk].ravel(), Fh[pk].ravel(), np.zeros(2 * ns), P["mu"],
                             P["tol_temp"], winsize=w, winsize_list=np.stack([wl_np[pk], wl_np[pk]], 1),
                             nthreads=threads)
                t_solve = time.perf_counter() - t0
                if t_sp2_cpu is None:  # one global step on the whole mesh (single-threaded either way)
                    t1 = time.perf_counter()
                    O.subpb2_quadtree(coords_np, E_np, 2, betas[1], P["mu"], Uh.ravel(), Fh.ravel(), dirichlet=dir_np)
                    t_sp2_cpu = time.perf_counter() - t1
                t_global = t_sp2_cpu * n_global
            t_step = t_search + t_solve * n / ns + t_global
            per = (solves if quad else (counted if counted is not None else n)) / t_step
            key = "value" if threads > 1 else "value_1core"
            cpu[key] = per
            if threads > 1:
                cpu["cores"] = threads
        cpu["sample"] = ("whole-field search timed on a sample of grid subsets and scaled to the grid; "
                         "solves timed on 900 (150 on one core) mesh nodes and scaled to the mesh"
                         + ("; one global step on the whole mesh (element loop + sparse direct solve), times "
                            "the frame's global solves" if quad else ""))
    line = {"metric": METRIC if not quad else ("subset solves/s (1 LocalICGNQuadtree + 2 Subpb1Quadtree per node, "
                                               "with the frame's Subpb2Quadtree global solves)"),
            "value": (counted if (counted is not None and not quad) else solves) / (ms_step * 1e-3),
            "unit": UNIT if not quad else "subset solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 solve)", "data": "synthetic (seeded analytic speckle rendering)",
            "config": {"workload": args.workload, "subsets": int(n), "image": [int(M), int(N)], **P,
                       **({"elements": int(E_np.shape[0]), "hanging_nodes": int((E_np[:, 4:] > 0).sum()),
                           "dirichlet_nodes": int(np.size(dir_np)), "global_solves": int(n_global)} if quad else {})},
            "gpu_launches": int(launches), "clocks": clk, "verification": ver, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    ctx.close()


def run_sequence(args, P):
    """sequence4096 (without the learned initial guess): 50 stereo frame
    pairs at 4096 x 3000 uint16 with the stereo rig of the stereo2048 workload aimed at a plane stretched
    progressively (8 % in x at the last frame) with a growing local bulge, rendered on the GPU.
    Frame 0: stereo L0 -> R0 whole-field search + IC-GN (set-up, timed separately).  Frames
    1..49, each timed alone: temporal L0 -> Lk and R0 -> Rk IC-GN on the left mesh and the
    stereo-matched right mesh, from the previous frames' results (frame 1: whole-field
    search), and FP64 triangulation.  Every frame is checked on the FP64 oracle (a sample
    of subsets per camera from the device's own initial guesses) and against the rendering's
    ground truth."""
    import torch

    import aldic_b200 as A
    from aldic_b200 import synth, synth_gpu

    T = torch
    dev = T.device("cuda:0")
    T.cuda.set_device(dev)
    f64 = dict(dtype=T.float64, device=dev)
    t0 = time.perf_counter()
    sc = synth_gpu.stereo_sequence(frames=P["frames"], M=P["M"], N=P["N"], seed=args.seed + 3)
    T.cuda.synchronize(dev)
    render_s = time.perf_counter() - t0
    M, N, K = sc.M, sc.N, P["frames"]
    w, st = P["w"], P["step"]
    gx, gy, shp = [1, M], [1, N], (M, N)
    coords_np, nx, ny = grid_coords(M, N, w, st)
    n, g = coords_np.shape[0], nx * ny
    coords = T.from_numpy(np.ascontiguousarray(coords_np.T)).to(dev)
    cxy = coords.t()
    sL, sR = T.cuda.Stream(dev), T.cuda.Stream(dev)
    cS, cL, cR = A.Context(0), A.Context(0), A.Context(0)
    cS.set_stream(sL.cuda_stream)
    cL.set_stream(sL.cuda_stream)
    cR.set_stream(sR.cuda_stream)

    def grid_buf():
        return {nm: T.empty(g, **f64) for nm in ("x", "y", "u", "v", "phi")}

    def icgn_buf():
        return {"U": T.empty(2 * n, **f64), "F": T.empty(4 * n, **f64), "conv": T.empty(n, dtype=T.int32, device=dev)}

    def grid_to_U0(b, ctx):
        """funRemoveOutliers(u, v, cc, 0, 100), then Init(u, v, Phi, x, y, 0) on the device:
        the search grids inpainted, mesh order."""
        out = T.empty(2 * g, **f64)
        ctx.remove_outliers(b["u"].view(nx, ny), b["v"].view(nx, ny), 100.0)
        ctx.init_u0(b["u"].view(nx, ny), b["v"].view(nx, ny), out=out)
        return out

    # ---- frame 0: stereo match (set-up) ----
    bS, oS = grid_buf(), icgn_buf()
    U0S = T.empty(2 * n, **f64)
    e0, e1 = T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True)
    with T.cuda.stream(sL):
        e0.record(sL)
        cS.load_image_raw(0, sc.L[0], gx, gy, want_stats=False, shape=shp)
        cS.load_image_raw(1, sc.R[0], gx, gy, want_stats=False, shape=shp)
        cS.compute_gradients()
        cS.integer_search(list(P["s_stereo"]), gx, gy, w, st, out=bS)
        U0S.copy_(grid_to_U0(bS, cS))
        cS.local_icgn(1, coords, U0S, w, P["tol_stereo"], out=oS)
        e1.record(sL)
    T.cuda.synchronize(dev)
    stereo_ms = e0.elapsed_time(e1)
    US = T.nan_to_num(oS["U"].view(n, 2), nan=0.0)
    coordsR = (cxy + US).t().contiguous()
    # temporal contexts keep frame 0 as the reference (slot 0) and its gradients
    with T.cuda.stream(sL):
        cL.load_image_raw(0, sc.L[0], gx, gy, want_stats=False, shape=shp)
        cL.compute_gradients()
    with T.cuda.stream(sR):
        cR.load_image_raw(0, sc.R[0], gx, gy, want_stats=False, shape=shp)
        cR.compute_gradients()
    T.cuda.synchronize(dev)
    bL1, bR1 = grid_buf(), grid_buf()
    res = {cam: [icgn_buf() for _ in range(K)] for cam in ("L", "R")}
    U0s = {cam: [T.zeros(2 * n, **f64) for _ in range(K)] for cam in ("L", "R")}
    xyz = [{"xyz": T.empty(3 * n, **f64), "err": T.empty(n, **f64)} for _ in range(2)]
    pairs = T.empty((4, n), **f64)
    for cam in ("L", "R"):
        res[cam][0]["U"].zero_()
        res[cam][0]["conv"].fill_(1)

    def init_guess(cam, k, ctx, crd, gb):
        """U0 of frame k: frame 1 from a whole-field search, later frames by extrapolating the
        last two results (a subset without both falls back to the last finite one, then 0)."""
        if k == 1:
            ctx.integer_search([P["s_temp"]] * 2, gx, gy, w, st, out=gb)
            Ug = grid_to_U0(gb, ctx)
            if crd is None:
                return Ug
            xy = crd.t()
            i = T.clamp(T.round((xy[:, 0] - (1 + w / 2.0)) / st), 0, nx - 1).long()
            j = T.clamp(T.round((xy[:, 1] - (1 + w / 2.0)) / st), 0, ny - 1).long()
            return Ug.view(-1, 2)[i + j * nx].reshape(-1)
        a, b = res[cam][k - 1]["U"], res[cam][k - 2]["U"]
        ext = 2 * a - b
        return T.where(T.isfinite(ext), ext, T.where(T.isfinite(a), a, T.zeros_like(a)))

    def frame(k):
        start, done_r, end = (T.cuda.Event(enable_timing=True) for _ in range(3))
        start.record(sL)
        sR.wait_event(start)
        with T.cuda.stream(sL):
            cL.load_image_raw(1, sc.L[k], gx, gy, want_stats=False, shape=shp)
            U0s["L"][k].copy_(init_guess("L", k, cL, None, bL1))
            cL.local_icgn(1, coords, U0s["L"][k], w, P["tol_temp"], out=res["L"][k])
        with T.cuda.stream(sR):
            cR.load_image_raw(1, sc.R[k], gx, gy, want_stats=False, shape=shp)
            U0s["R"][k].copy_(init_guess("R", k, cR, coordsR, bR1))
            cR.local_icgn(1, coordsR, U0s["R"][k], w, P["tol_temp"], out=res["R"][k])
            done_r.record(sR)
        with T.cuda.stream(sL):
            sL.wait_event(done_r)
            UL, UR = res["L"][k]["U"].view(n, 2), res["R"][k]["U"].view(n, 2)
            pairs.copy_(T.cat([cxy + UL, coordsR.t() + UR], 1).t())
            cS.triangulate(pairs, sc.KL, sc.KR, sc.R_rl, sc.T_rl, out=xyz[k % 2])
            end.record(sL)
        return start, end

    # warm-up: the first frames once (the timed pass starts the sequence again)
    for k in range(1, 1 + max(args.warmup, 3)):
        frame(k)
    T.cuda.synchronize(dev)
    clocks = ClockSampler(0)
    l0 = cS.launches + cL.launches + cR.launches
    evs = [frame(k) for k in range(1, K)]
    T.cuda.synchronize(dev)
    clk = clocks.stop()
    launches = cS.launches + cL.launches + cR.launches - l0
    lat = np.array([a.elapsed_time(b) for a, b in evs])
    total_ms = evs[0][0].elapsed_time(evs[-1][1])
    conv = {cam: np.stack([res[cam][k]["conv"].cpu().numpy() for k in range(K)]) for cam in ("L", "R")}
    converged = sum(int(((conv[c][1:] > 0) & (conv[c][1:] < 100)).sum()) for c in ("L", "R"))

    # ---- verification on the FP64 oracle and the rendering's ground truth (untimed) ----
    import oracle as O

    O.build()
    nthr = host_threads()
    rng = np.random.default_rng(5)
    m = min(P["sample"], n)
    pick = np.sort(rng.choice(n, m, replace=False))
    crdL = coords_np[pick]
    crdR = coordsR.t().cpu().numpy()[pick]

    def host(img):
        return img.to(T.int32).cpu().numpy().reshape(N, M).T.astype(np.float64)

    def norm(img):
        return O.normalize(host(img), gx, gy)[0]

    fL0, fR0 = norm(sc.L[0]), norm(sc.R[0])
    gL0, gR0 = O.gradient(fL0), O.gradient(fR0)
    # stereo: IC-GN from the device's initial guesses, and the whole-field search on a few subsets
    o = O.local_icgn(O.Frame(fL0, fR0, None, gL0[0], gL0[1]), crdL, U0S.view(n, 2)[pick].cpu().numpy().ravel(), w,
                     P["tol_stereo"], variant=1, nthreads=nthr)
    cg = oS["conv"].cpu().numpy()[pick]
    fg_d, fg_o = (cg > 0) & (cg < 100), (o["conv"] > 0) & (o["conv"] < 100)
    both = fg_d & fg_o
    dU = np.abs(oS["U"].view(n, 2).cpu().numpy()[pick] - o["U"].reshape(-1, 2)).max(1)
    qs = pick[:12]
    pi, pj = qs % nx, qs // nx  # mesh order: XList fastest
    sub = O.search_list(fL0, fR0, list(P["s_stereo"]), M, N, 1 + pi * st, 1 + pj * st, w, nthreads=nthr)
    gu = bS["u"].cpu().numpy().reshape(nx, ny).T
    gv = bS["v"].cpu().numpy().reshape(nx, ny).T
    same = (sub[:, 0] == gu[pj, pi]) & (sub[:, 1] == gv[pj, pi])
    same |= np.isnan(sub[:, 0]) & np.isnan(gu[pj, pi])
    stereo_ver = {"sample": m, "flag_match": float(np.mean(fg_d == fg_o)),
                  "uv_max_err": float(dU[both].max()) if both.any() else None,
                  "search_sample_exact": f"{int(same.sum())}/{len(qs)}",
                  "converged": int(((oS["conv"] > 0) & (oS["conv"] < 100)).sum())}
    # temporal frames: every frame, both cameras
    W0 = synth._ray_plane(sc.camL, crdL[:, 0], crdL[:, 1], sc.Z)  # frame-0 plane = material coordinates
    per = {"flag_match": [], "uv_max_err": [], "truth_median_err": [], "truth_p95_err": []}
    t_oracle, n_oracle = 0.0, 0
    for k in range(1, K):
        wk = sc.material_to_world(W0[:, 0], W0[:, 1], k)
        uu, vv = sc.camL.project(wk)
        Utrue = np.stack([uu + 1.0, vv + 1.0], 1) - crdL
        fmk, emk = [], []
        for cam, f0, g0, crd in (("L", fL0, gL0, crdL), ("R", fR0, gR0, crdR)):
            gk = norm((sc.L if cam == "L" else sc.R)[k])
            ta = time.perf_counter()
            o = O.local_icgn(O.Frame(f0, gk, None, g0[0], g0[1]), crd,
                             U0s[cam][k].view(n, 2)[pick].cpu().numpy().ravel(), w, P["tol_temp"], variant=1,
                             nthreads=nthr)
            t_oracle += time.perf_counter() - ta
            n_oracle += m
            cd = res[cam][k]["conv"].cpu().numpy()[pick]
            Ud = res[cam][k]["U"].view(n, 2).cpu().numpy()[pick]
            fd, fo = (cd > 0) & (cd < 100), (o["conv"] > 0) & (o["conv"] < 100)
            fmk.append(float(np.mean(fd == fo)))
            bo = fd & fo
            if bo.any():
                emk.append(float(np.abs(Ud - o["U"].reshape(-1, 2)).max(1)[bo].max()))
            if cam == "L":
                e = np.abs(Ud - Utrue).max(1)[fd]
                per["truth_median_err"].append(round(float(np.median(e)), 4) if e.size else None)
                per["truth_p95_err"].append(round(float(np.percentile(e, 95)), 4) if e.size else None)
        per["flag_match"].append(min(fmk))
        per["uv_max_err"].append(max(emk) if emk else None)
    errs = [e for e in per["uv_max_err"] if e is not None]
    line = {
        "metric": "converged temporal IC-GN subsets/s over frames 1-49 (2 cameras), 4096x3000 stereo sequence",
        "value": converged / (total_ms * 1e-3), "unit": "subsets/s", "n_gpus": 1, "steps": K - 1,
        "warmup": max(args.warmup, 3), "ms_per_step": float(lat.mean()), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 solve/fit/triangulation)",
        "data": "synthetic (seeded analytic speckle rendering on the GPU)",
        "config": {"workload": "sequence4096", "subsets_per_camera": n, "frames": K,
                   "init": "frame 1: whole-field search [10 10]; frames 2-49: extrapolation of the last two "
                           "results; no learned initial guess",
                   "l2_flush": "each frame reads new 24 MB frames and 0.5 GB of per-context images / gradients",
                   **{k: v for k, v in P.items() if k != "sample"}},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "stereo_frame0": stereo_ms},
        "gpu_launches": int(launches),
        "cpu_baseline": {"value": n_oracle / t_oracle if t_oracle else None, "unit": "subsets/s", "cores": nthr,
                         "kind": "port",
                         "sample": f"FP64 oracle IC-GN on {m} subsets per camera and frame from the device's own "
                                   f"initial guesses, frames 1-{K - 1}"},
        "clocks": clk,
        "verification": {"stereo_frame0": stereo_ver, "sample_per_camera": m,
                         "temporal_flag_match_min": min(per["flag_match"]),
                         "temporal_uv_max_err": max(errs) if errs else None,
                         "per_frame": per, "render_s": render_s,
                         "converged_fraction": converged / (2.0 * n * (K - 1))},
    }
    print(json.dumps(line), flush=True)
    for c in (cS, cL, cR):
        c.close()

def measure_fp32_peak(torch, dev):
    import aldic_b200 as A

    lib = A.load_library()
    if not hasattr(lib, "aldic_measure_fp32_peak"):
        return None
    import ctypes as C

    c = A.Context(dev.index or 0)
    out = C.c_double()
    rc = lib.aldic_measure_fp32_peak(c.h, C.byref(out))
    c.close()
    return out.value if rc == 0 else None


def e2e_measure(A, scene, P, steps, local_rank):
    """The same pass through the public API with host buffers: every call copies its
    inputs host->device and its results device->host.  Frames and result buffers live in
    pinned host memory; the three passes run as host threads on their own contexts (and
    so their own streams), the way a caller overlaps independent passes; the right
    temporal pass waits for the stereo result before its IC-GN."""
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch

    M = N = P["size"]
    w, st = P["w"], P["step"]
    coords, nx, ny = grid_coords(M, N, w, st)
    n, g = coords.shape[0], nx * ny

    def pinned(shape, dtype=np.float64, order="C"):
        shape = (shape,) if np.isscalar(shape) else tuple(shape)
        nb = int(np.prod(shape)) * np.dtype(dtype).itemsize
        raw = torch.empty(nb, dtype=torch.uint8, pin_memory=True).numpy()
        return raw.view(dtype).reshape(shape, order=order)

    imgs = {}
    for k, v in (("L0", scene.L[0]), ("L1", scene.L[1]), ("R0", scene.R[0]), ("R1", scene.R[1])):
        imgs[k] = pinned(v.shape, v.dtype, order="F")
        imgs[k][...] = v
    ctx = {k: A.Context(local_rank) for k in ("S", "L", "R")}
    for c in ctx.values():
        c.set_option(A.OPT_AUTOTUNE, 1)  # tuned in the warm-up pass, as the device pipeline
    # the step's results: U, F and the convergence codes (the per-subset Hessian H is an
    # input of ALDIC's Subpb1 step only, which this pipeline does not run, so it is not read)
    out = {k: {**{nm: pinned(g) for nm in ("x", "y", "u", "v", "phi")},
               "U": pinned(2 * n), "F": pinned(4 * n), "conv": pinned(n, np.int32)}
           for k in ("S", "L", "R")}
    tri = [{"xyz": pinned(3 * n), "err": pinned(n)} for _ in range(2)]
    U0 = {k: pinned(2 * n) for k in ("S", "L", "R")}
    Ug = pinned(2 * g)
    # MATLAB column-major n x 2 / n x 4 arrays: the library reads them without a repack
    crd = pinned((n, 2), order="F")
    crd[:] = coords
    crdR = pinned((n, 2), order="F")
    pairs = [pinned((n, 4), order="F") for _ in range(2)]
    gx, gy = [1, M], [1, N]
    grid_bytes = 5 * g * 8
    icgn_out_bytes = (2 + 4) * n * 8 + n * 4

    def search(k, ref, cur, s, after=None):
        c, o = ctx[k], out[k]
        c.load_image_raw(0, imgs[ref], gx, gy, want_stats=False)
        c.load_image_raw(1, imgs[cur], gx, gy, want_stats=False)
        c.compute_gradients()
        if after is not None:  # the temporal searches wait for the stereo search, as on the device
            after.wait()
        c.integer_search([s, s], gx, gy, w, st, out=o)
        return o["u"].reshape((ny, nx), order="F"), o["v"].reshape((ny, nx), order="F")

    stereo_done = threading.Event()
    search_done = threading.Event()

    def stereo():
        u, v = search("S", "L0", "R0", P["s_stereo"])
        search_done.set()
        u, v = ctx["S"].remove_outliers(u, v, 100.0)
        ctx["S"].init_u0(u, v, out=U0["S"])
        ctx["S"].local_icgn(1, crd, U0["S"], w, P["tol_stereo"], out=out["S"])
        stereo_done.set()

    def left():
        u, v = search("L", "L0", "L1", P["s_temp"], after=search_done)
        u, v = ctx["L"].remove_outliers(u, v, 100.0)
        ctx["L"].init_u0(u, v, out=U0["L"])
        ctx["L"].local_icgn(1, crd, U0["L"], w, P["tol_temp"], out=out["L"])

    def right():
        u, v = search("R", "R0", "R1", P["s_temp"], after=search_done)
        u, v = ctx["R"].remove_outliers(u, v, 100.0)
        stereo_done.wait()
        # right-camera mesh = left mesh + stereo match; initial guess: Init over the search
        # grid, then the nearest grid node of each right-image point
        ctx["R"].init_u0(u, v, out=Ug)
        crdR[:] = coords + np.nan_to_num(out["S"]["U"].reshape(n, 2))
        i = np.clip(np.round((crdR[:, 0] - (1 + w / 2.0)) / st), 0, nx - 1).astype(int)
        j = np.clip(np.round((crdR[:, 1] - (1 + w / 2.0)) / st), 0, ny - 1).astype(int)
        U0["R"].reshape(n, 2)[:] = Ug.reshape(-1, 2)[i + j * nx]
        ctx["R"].local_icgn(1, crdR, U0["R"], w, P["tol_temp"], out=out["R"])

    pool = ThreadPoolExecutor(3)
    conv_total = 0

    def one():
        nonlocal conv_total
        stereo_done.clear()
        search_done.clear()
        for f in [pool.submit(fn) for fn in (stereo, left, right)]:
            f.result()
        US, UL, UR = (out[k]["U"].reshape(n, 2) for k in ("S", "L", "R"))
        pairs[0][:, :2] = coords
        pairs[0][:, 2:] = coords + US
        pairs[1][:, :2] = coords + UL
        pairs[1][:, 2:] = coords + US + UR
        for p, o in zip(pairs, tri):
            ctx["S"].triangulate(p, scene.KL, scene.KR, scene.R_rl, scene.T_rl, out=o)
        conv_total += sum(int(np.sum((out[k]["conv"] > 0) & (out[k]["conv"] < 100))) for k in ("S", "L", "R"))
        # per pass: the grids staged through the bad-point removal (2 g doubles each way), then
        # through Init (2 g in, U0 out), the mesh, the IC-GN outputs
        h2d = 6 * imgs["L0"].nbytes + 3 * (2 * n * 8 + U0["S"].nbytes + 4 * g * 8) + 2 * pairs[0].nbytes
        d2h = 3 * (grid_bytes + icgn_out_bytes + 4 * g * 8) + 2 * (tri[0]["xyz"].nbytes + tri[0]["err"].nbytes)
        return h2d, d2h

    one()  # warm-up
    conv_total = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        h2d, d2h = one()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1000 / steps
    pool.shutdown()
    for c in ctx.values():
        c.close()
    return {"ms": ms, "converged": conv_total / steps, "h2d": h2d, "d2h": d2h}


if __name__ == "__main__":
    main()
