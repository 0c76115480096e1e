"""The learned initial guess: host side of the proposal network (csrc/cnn.cu).

The network reads a 32 x 32 reference subset and the 64 x 64 deformed window around it (with
4 px of context each side: a 72 x 72 x 2 input) and predicts (u, v, du/dx, dv/dx, du/dy, dv/dy) as IC-GN's initial guess [F0 U0], in place of the
integer search (func/funIntegerSearch.m:132-180), which stays the fallback and the judge.  It
has no counterpart in the reference.  Everything here drives the library's C ABI: device
memory comes from torch, every layer, gradient and optimiser step is the library's own
kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import AldicError

SCALE = np.array([1 / 8.0, 1 / 8.0, 20.0, 20.0, 20.0, 20.0], dtype=np.float32)  # network output units


# weight matrices (rows x cols, row-major, then rows biases) of the four 3 x 3 convolutions
# (cols = 9 x input channels, padded to a multiple of 8: conv1 9 -> 16, conv3 729 -> 736) and
# the two fully connected layers (1024 -> 128 -> 6, the output padded to 16 rows)
_ROWS = (32, 32, 64, 64, 128, 16)
_COLS = (16, 288, 736, 576, 1024, 128)
_FAN_IN = (9, 288, 729, 576, 1024, 128)


def param_count():
    return int(_lib.load().aldic_net_param_count())


def init_params(seed=0):
    """He-normal weights (std sqrt(2 / fan-in)) and zero biases, with the padding columns of
    the convolutions and the padding rows of the output layer zero: the flat FP32 vector
    aldic_net_set_params takes."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (r, c) in enumerate(zip(_ROWS, _COLS)):
        W = rng.normal(0.0, np.sqrt(2.0 / _FAN_IN[l]), (r, c)).astype(np.float32)
        W[:, _FAN_IN[l]:] = 0.0
        if l == len(_ROWS) - 1:
            W[6:, :] = 0.0
        parts += [W.ravel(), np.zeros(r, dtype=np.float32)]
    p = np.concatenate(parts)
    if p.size != param_count():
        raise AldicError(f"parameter layout mismatch: {p.size} vs {param_count()}")
    return p


class ProposalNet:
    """The network on one device: FP32 parameters (He-normal from `seed`) with BF16 copies,
    Adam moments and the activation buffers of batches up to max_batch (a multiple of 8)."""

    def __init__(self, device=0, max_batch=256, seed=0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.aldic_net_create(C.byref(h), int(device), int(max_batch))
        if rc != _lib.ALDIC_OK:
            raise AldicError(f"aldic_net_create failed ({rc})")
        self.h = h
        self.max_batch = max_batch
        self.n_params = param_count()
        self.set_params(init_params(seed))

    def close(self):
        if self.h:
            self.lib.aldic_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != _lib.ALDIC_OK:
            raise AldicError(f"{what}: {self.lib.aldic_net_last_error(self.h).decode()}")

    @property
    def launches(self):
        return int(self.lib.aldic_net_launch_count(self.h))

    def set_stream(self, handle):
        self._check(self.lib.aldic_net_set_stream(self.h, C.c_void_p(handle)), "aldic_net_set_stream")

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise AldicError(f"{p.size} parameters, {self.n_params} expected")
        self._check(self.lib.aldic_net_set_params(self.h, C.c_void_p(p.ctypes.data)), "aldic_net_set_params")

    def get_params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        self._check(self.lib.aldic_net_get_params(self.h, C.c_void_p(p.ctypes.data)), "aldic_net_get_params")
        return p

    @staticmethod
    def _dev(t, dtype, shape_tail):
        if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous()):
            raise AldicError("network inputs are contiguous CUDA tensors")
        if str(t.dtype) != dtype or tuple(t.shape[1:]) != shape_tail:
            raise AldicError(f"expected {dtype} (batch, {shape_tail}), got {t.dtype} {tuple(t.shape)}")
        return C.c_void_p(t.data_ptr())

    def forward(self, x, out):
        """out (batch, 6) float32 CUDA tensor <- the scaled outputs for x (batch, 72, 72, 2) bf16."""
        b = int(x.shape[0])
        self._check(self.lib.aldic_net_forward(self.h, b, self._dev(x, "torch.bfloat16", (72, 72, 2)),
                                               self._dev(out, "torch.float32", (6,))), "aldic_net_forward")
        return out

    def gradients(self, x, t):
        """(loss, flat FP32 gradients) of the mean squared error against t (batch, 6)."""
        g = np.empty(self.n_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.aldic_net_gradients(self.h, int(x.shape[0]), self._dev(x, "torch.bfloat16", (72, 72, 2)),
                                                 self._dev(t, "torch.float32", (6,)), C.c_void_p(g.ctypes.data),
                                                 C.c_void_p(loss.ctypes.data)), "aldic_net_gradients")
        return float(loss[0]), g

    def train_step(self, x, t, lr, want_loss=False):
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.aldic_net_train_step(self.h, int(x.shape[0]), self._dev(x, "torch.bfloat16", (72, 72, 2)),
                                                  self._dev(t, "torch.float32", (6,)), C.c_float(lr),
                                                  C.c_void_p(loss.ctypes.data) if want_loss else None),
                    "aldic_net_train_step")
        return float(loss[0]) if want_loss else None

    def status(self):
        self._check(self.lib.aldic_net_status(self.h), "aldic_net_status")

    def predict(self, ctx, coords, out):
        """Initial guesses of the subsets at coords (a (2, n) float64 CUDA tensor: the MATLAB
        n x 2 layout) on ctx's frame into out["U0"] (2n) and out["F0"] (4n) CUDA tensors."""
        n = int(coords.shape[1])
        rc = self.lib.aldic_net_predict(self.h, ctx.h, n, C.c_void_p(coords.data_ptr()),
                                        C.c_void_p(out["U0"].data_ptr()), C.c_void_p(out["F0"].data_ptr()))
        ctx._check(rc, "aldic_net_predict")
        return out


def gemm_bf16(A, B, C_out, splits=1, stream=0):
    """C_out (M x N float32) = A (M x K bf16) B (N x K bf16)^T on the tensor cores."""
    lib = _lib.load()
    M, K = A.shape
    N = B.shape[0]
    rc = lib.aldic_gemm_bf16(C.c_void_p(A.data_ptr()), A.stride(0), C.c_void_p(B.data_ptr()), B.stride(0), M, N, K,
                             C.c_void_p(C_out.data_ptr()), C_out.stride(0), int(splits), C.c_void_p(stream))
    if rc != _lib.ALDIC_OK:
        raise AldicError(f"aldic_gemm_bf16 failed ({rc})")
    return C_out


# ------------------------------------------------------------------------ training
def grid_nodes(M, N, w, step, margin=None):
    """Subset centres (1-based) of a uniform grid whose 72 x 72 network windows stay inside the
    image: a (2, n) float64 array, x fastest."""
    m = 37 if margin is None else margin
    lo = max(m, w // 2 + 4)
    xs = np.arange(lo, M - lo + 1, step, dtype=np.float64)
    ys = np.arange(lo, N - lo + 1, step, dtype=np.float64)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    return np.stack([X.ravel(order="F"), Y.ravel(order="F")], 0)


def label_pair(ctx, pair, w=32, step=12, tol=1e-3, variant=_lib.QUADTREE, stream=None, umax=12.0):
    """Training samples of one speckle pair (synth_gpu.FieldPair): the network inputs of the
    pair's own nodes (a tile mosaic's tile centres) or of a grid of subsets whose 72 x 72
    windows lie inside the image, whose displacement is within umax, and, as labels, the method's own converged IC-GN results (LocalICGN's loop body
    started from the field's analytic displacement and gradient); unconverged subsets are
    dropped.  Returns CUDA tensors X bf16
    (n, 72, 72, 2) and T float32 (n, 6) (scaled outputs), made on `stream` (a torch stream;
    a new one if None) which the current stream then waits for."""
    import torch as T

    st = stream or T.cuda.Stream()
    ctx.set_stream(st.cuda_stream)
    M, N = pair.M, pair.N
    with T.cuda.stream(st):
        ctx.load_image_raw(0, pair.ref, [1, M], [1, N], want_stats=False, shape=(M, N))
        ctx.load_image_raw(1, pair.deff, [1, M], [1, N], want_stats=False, shape=(M, N))
        ctx.compute_gradients()
        nodes = getattr(pair, "nodes", None)
        if nodes is None:
            nodes = grid_nodes(M, N, w, step)
        u, v = pair.field.disp(nodes[0], nodes[1])
        keep = (np.abs(u) <= umax) & (np.abs(v) <= umax)
        nodes, u, v = nodes[:, keep], u[keep], v[keep]
        U0 = np.stack([u, v], 1).ravel()
        F0 = pair.field.grad(nodes[0], nodes[1]).ravel()
        r = ctx.local_icgn(variant, nodes.T, U0, w, tol, F0=F0, want_H=False, want_mark=False)
        ok = (r["conv"] > 0) & (r["conv"] < 100)
        crd = T.from_numpy(np.ascontiguousarray(nodes[:, ok])).to(pair.ref.device, non_blocking=False)
        X = T.empty((int(ok.sum()), 72, 72, 2), dtype=T.bfloat16, device=pair.ref.device)
        ctx.net_extract(crd, X)
        lab = np.concatenate([r["U"].reshape(-1, 2)[ok], r["F"].reshape(-1, 4)[ok]], 1) * SCALE
        Tg = T.from_numpy(lab.astype(np.float32)).to(pair.ref.device)
    T.cuda.current_stream().wait_stream(st)
    return X, Tg


def train(net, X, Tgt, steps, batch=256, lr=1e-3, lr_end=1e-5, seed=0, log_every=100):
    """Adam steps on random minibatches of (X, Tgt) with a cosine learning-rate decay from lr to
    lr_end, on a stream of their own; returns the logged (step, loss) pairs."""
    import torch as T

    st = T.cuda.Stream(X.device)
    st.wait_stream(T.cuda.current_stream())
    net.set_stream(st.cuda_stream)
    gen = T.Generator(device=X.device)
    gen.manual_seed(seed)
    n = X.shape[0]
    log = []
    with T.cuda.stream(st):
        for k in range(steps):
            idx = T.randint(0, n, (batch,), device=X.device, generator=gen)
            rate = lr_end + 0.5 * (lr - lr_end) * (1 + np.cos(np.pi * k / max(steps - 1, 1)))
            want = (k % log_every == 0) or k == steps - 1
            loss = net.train_step(X.index_select(0, idx), Tgt.index_select(0, idx), float(rate), want_loss=want)
            if want:
                log.append((k, loss))
    st.synchronize()
    net.set_stream(None)
    net.status()
    return log


# ------------------------------------------------------------------------ inference
def search_nodes(gridx, gridy, winsize, step):
    """Centres (1-based) of the integer-search grid subsets of funIntegerSearchWholeField
    (func/funIntegerSearch.m:132-180): x = gridx[0] + i step + winsize / 2 and y alike, in grid
    order t = i + j nX (MeshSetUp's coordinatesFEM order).  Returns ((2, n) float64, nX, nY)."""
    ex, ey = gridx[1] - winsize - step, gridy[1] - winsize - step
    nx = (ex - gridx[0]) // step + 1 if ex >= gridx[0] else 0
    ny = (ey - gridy[0]) // step + 1 if ey >= gridy[0] else 0
    xs = gridx[0] + step * np.arange(nx) + winsize / 2.0
    ys = gridy[0] + step * np.arange(ny) + winsize / 2.0
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    return np.stack([X.ravel(order="F"), Y.ravel(order="F")], 0), nx, ny


class LearnedInit:
    """IC-GN with the network's initial guess on the subsets of an integer-search grid, the
    integer search as the fallback and the judge.

    run() on the frame resident in ctx: the network predicts [F0 U0] for every grid subset,
    IC-GN (LocalICGN's loop body) runs from it, and a subset whose IC-GN did not converge or
    whose final ZNCC is below zncc_min is searched (funIntegerSearchWholeField restricted to
    those grid subsets) and solved again from the search's [0 U0], as the reference's
    search-initialised path would.  Everything stays on ctx's stream; the host waits once, for
    the number of fallback subsets.  run() = submit() (queue the frame) + complete() (that
    wait, then queue the fallback); LearnedPipeline puts another frame between the two."""

    def __init__(self, net, ctx, search, gridx, gridy, winsize, step, tol, zncc_min=0.9, variant=_lib.QUADTREE,
                 stream=None):
        import torch as T

        self.T, self.net, self.ctx = T, net, ctx
        self.search = [int(search)] * 2 if np.ndim(search) == 0 else [int(s) for s in search]
        self.gx, self.gy = [int(g) for g in gridx], [int(g) for g in gridy]
        self.w, self.step, self.tol, self.zncc_min, self.variant = int(winsize), int(step), tol, zncc_min, variant
        nodes, self.nx, self.ny = search_nodes(self.gx, self.gy, self.w, self.step)
        self.n = n = nodes.shape[1]
        dev = T.device("cuda", ctx.device if hasattr(ctx, "device") else T.cuda.current_device())
        # one stream for everything (a given one lets several contexts share the network's
        # buffers in order, e.g. frames pipelined over two contexts)
        self.stream = stream if stream is not None else T.cuda.Stream(dev)
        ctx.set_stream(self.stream.cuda_stream)
        f64 = dict(dtype=T.float64, device=dev)
        self.coords = T.from_numpy(np.ascontiguousarray(nodes)).to(dev)
        self.buf = {"U0": T.empty(2 * n, **f64), "F0": T.empty(4 * n, **f64), "U": T.empty(2 * n, **f64),
                    "F": T.empty(4 * n, **f64), "conv": T.empty(n, dtype=T.int32, device=dev),
                    "zncc": T.empty(n, **f64), "fallback": T.zeros(n, dtype=T.bool, device=dev)}
        self.flist = T.empty(n, dtype=T.int32, device=dev)
        self.count_dev = T.zeros(1, dtype=T.int64, device=dev)
        self.count_host = T.zeros(1, dtype=T.int64, pin_memory=True)
        self.count_event = T.cuda.Event()
        self.n_fallback = 0
        # (start, stop) CUDA event pairs recorded around the prediction and the main IC-GN call
        # when these are lists (timing hooks)
        self.predict_events = None
        self.icgn_events = None

    def _timed(self, events, fn):
        if events is None:
            return fn()
        T = self.T
        e = (T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True))
        e[0].record(self.stream)
        r = fn()
        e[1].record(self.stream)
        events.append(e)
        return r

    def run(self):
        """One frame; returns the number of fallback subsets."""
        self.submit()
        return self.complete()

    def submit(self):
        """Queue one frame on the stream without waiting: prediction, IC-GN from [F0 U0] (its
        last iteration's sums give each subset's ZNCC) and the fallback selection, whose count
        is copied to pinned host memory.  complete() finishes the frame; a caller may queue
        another frame (on another context) in between."""
        T, ctx, b = self.T, self.ctx, self.buf
        with T.cuda.stream(self.stream):
            self._timed(self.predict_events, lambda: self.net.predict(ctx, self.coords, b))
            self._timed(self.icgn_events,
                        lambda: ctx.local_icgn(self.variant, self.coords, b["U0"], self.w, self.tol, want_H=False,
                                               want_mark=False, out=b, F0=b["F0"], want_zncc=True))
            ctx.fallback_select(b["conv"], b["zncc"], self.zncc_min, self.flist, count=self.count_dev)
            self.count_host.copy_(self.count_dev, non_blocking=True)
            self.count_event.record(self.stream)

    def complete(self):
        """Wait for the submitted frame's fallback count (the host's one wait per frame) and
        queue the fallback: the integer search on those grid subsets and IC-GN from its
        [0 U0].  Returns the number of fallback subsets."""
        T, ctx, b, n = self.T, self.ctx, self.buf, self.n
        self.count_event.synchronize()
        nf = int(self.count_host[0])
        with T.cuda.stream(self.stream):
            b["fallback"].zero_()
            if nf:
                il = self.flist[:nf]
                idx = il.long()
                b["fallback"][idx] = True
                dev = self.coords.device
                f64 = dict(dtype=T.float64, device=dev)
                r = {k: T.empty(nf, **f64) for k in ("x", "y", "u", "v", "phi")}
                ctx.integer_search_list(self.search, self.gx, self.gy, self.w, self.step, il, out=r)
                U0f = T.nan_to_num(T.stack([r["u"], r["v"]], 1), nan=0.0).reshape(-1).contiguous()
                crd = self.coords.index_select(1, idx).contiguous()
                o = {"U": T.empty(2 * nf, **f64), "F": T.empty(4 * nf, **f64),
                     "conv": T.empty(nf, dtype=T.int32, device=dev)}
                ctx.local_icgn(self.variant, crd, U0f, self.w, self.tol, want_H=False, want_mark=False, out=o)
                b["U"].view(n, 2)[idx] = o["U"].view(nf, 2)
                b["F"].view(n, 4)[idx] = o["F"].view(nf, 4)
                b["conv"][idx] = o["conv"]
                b["U0"].view(n, 2)[idx] = U0f.view(nf, 2)
                b["F0"].view(n, 4)[idx] = 0.0
        self.n_fallback = nf
        return nf


class LearnedPipeline:
    """Frames through the learned initial guess with two contexts in flight: frame k is loaded
    into one context and queued (LearnedInit.submit) before the host waits for frame k-1's
    fallback count (LearnedInit.complete), so that wait, and the host's launches of frame k,
    overlap the device's work instead of leaving it idle.  Both LearnedInit objects share the
    network and one stream (the network's buffers are used in stream order).  Arguments after
    `ctxs` (two contexts on the same device) are LearnedInit's."""

    def __init__(self, net, ctxs, *args, **kw):
        if len(ctxs) != 2:
            raise ValueError("LearnedPipeline takes two contexts")
        first = LearnedInit(net, ctxs[0], *args, **kw)
        kw = dict(kw, stream=first.stream)
        self.lis = [first, LearnedInit(net, ctxs[1], *args, **kw)]
        self.stream = first.stream
        self.turn = 0
        self.pending = None

    def push(self, load):
        """load(ctx) queues the next frame's images into a context (on the stream); the frame
        is then submitted and the previous one completed.  Returns the LearnedInit that holds
        the previous frame's results (valid on the stream until the push after next), or None
        for the first frame."""
        import torch as T

        li = self.lis[self.turn]
        self.turn ^= 1
        with T.cuda.stream(self.stream):
            load(li.ctx)
        li.submit()
        done, self.pending = self.pending, li
        if done is not None:
            done.complete()
        return done

    def flush(self):
        """Completes the last pushed frame; returns its LearnedInit (or None)."""
        done, self.pending = self.pending, None
        if done is not None:
            done.complete()
        return done
