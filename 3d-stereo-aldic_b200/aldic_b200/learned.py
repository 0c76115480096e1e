"""The learned initial guess: host side of the proposal network (csrc/cnn.cu).

The network reads a 32 x 32 reference subset and the 64 x 64 deformed window around it and
predicts (u, v, du/dx, dv/dx, du/dy, dv/dy) as IC-GN's initial guess [F0 U0], in place of the
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


def param_count():
    return int(_lib.load().aldic_net_param_count())


class ProposalNet:
    """The network on one device: FP32 parameters with BF16 copies, Adam moments and the
    activation buffers of batches up to max_batch (a multiple of 8)."""

    def __init__(self, device=0, max_batch=256):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.aldic_net_create(C.byref(h), int(device), int(max_batch))
        if rc != _lib.ALDIC_OK:
            raise AldicError(f"aldic_net_create failed ({rc})")
        self.h = h
        self.max_batch = max_batch
        self.n_params = param_count()

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
        """out (batch, 6) float32 CUDA tensor <- the scaled outputs for x (batch, 64, 64, 2) bf16."""
        b = int(x.shape[0])
        self._check(self.lib.aldic_net_forward(self.h, b, self._dev(x, "torch.bfloat16", (64, 64, 2)),
                                               self._dev(out, "torch.float32", (6,))), "aldic_net_forward")
        return out

    def gradients(self, x, t):
        """(loss, flat FP32 gradients) of the mean squared error against t (batch, 6)."""
        g = np.empty(self.n_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.aldic_net_gradients(self.h, int(x.shape[0]), self._dev(x, "torch.bfloat16", (64, 64, 2)),
                                                 self._dev(t, "torch.float32", (6,)), C.c_void_p(g.ctypes.data),
                                                 C.c_void_p(loss.ctypes.data)), "aldic_net_gradients")
        return float(loss[0]), g

    def train_step(self, x, t, lr, want_loss=False):
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.aldic_net_train_step(self.h, int(x.shape[0]), self._dev(x, "torch.bfloat16", (64, 64, 2)),
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
