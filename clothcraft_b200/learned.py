"""Learned initial guess: the MLP handle over the C ABI (cc_mlp_*).

Device arrays are CUDA float32 torch tensors (torch is only the allocator
here); every computation runs in the library's own kernels: FP32 or
tensor-core (FP16/FP32-accumulate) inference, FP32 forward/backward and Adam
for training. No reference counterpart: the reference always starts a step
from Prediction::guess (src/vbd/prediction.rs:15-41).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .vbd import VbdError

N_IN, N_HIDDEN, N_OUT = 24, 64, 3


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(t, cols):
    import torch

    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 2 and t.shape[1] == cols):
        raise ValueError("expected a contiguous CUDA float32 tensor [n, %d]" % cols)


class Mlp:
    """24-64-64-64-3 GELU network predicting the correction of the adaptive guess."""

    def __init__(self, seed: int = 0):
        L = native.load()
        h = C.c_void_p()
        rc = L.cc_mlp_create(int(seed), C.byref(h))
        if rc != 0:
            buf = C.create_string_buffer(1024)
            L.cc_global_last_error(buf, 1024)
            raise VbdError(rc, buf.value.decode())
        self.h = h
        self.count = int(L.cc_mlp_parameter_count())

    def __del__(self):
        if getattr(self, "h", None):
            native.load().cc_mlp_destroy(self.h)
            self.h = None

    def _err(self, rc):
        buf = C.create_string_buffer(1024)
        native.load().cc_mlp_last_error(self.h, buf, 1024)
        return VbdError(rc, buf.value.decode())

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.count, np.float32)
        rc = native.load().cc_mlp_get_parameters(self.h, _fp(out), self.count)
        if rc != 0:
            raise self._err(rc)
        return out

    def set_parameters(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32).ravel()
        rc = native.load().cc_mlp_set_parameters(self.h, _fp(p), p.size)
        if rc != 0:
            raise self._err(rc)

    def forward(self, features, precision: int = 0):
        import torch

        _check(features, N_IN)
        out = torch.empty((features.shape[0], N_OUT), dtype=torch.float32, device=features.device)
        torch.cuda.synchronize()
        rc = native.load().cc_mlp_forward(self.h, C.c_void_p(features.data_ptr()), features.shape[0],
                                          C.c_void_p(out.data_ptr()), int(precision))
        if rc != 0:
            raise self._err(rc)
        return out

    def gradients(self, features, targets):
        """(gradient [count], loss) of mean over samples of |MLP(f) - t|^2."""
        import torch

        _check(features, N_IN)
        _check(targets, N_OUT)
        g = np.zeros(self.count, np.float32)
        loss = C.c_float()
        torch.cuda.synchronize()
        rc = native.load().cc_mlp_gradients(self.h, C.c_void_p(features.data_ptr()), C.c_void_p(targets.data_ptr()),
                                            features.shape[0], _fp(g), C.byref(loss))
        if rc != 0:
            raise self._err(rc)
        return g, float(loss.value)

    def train(self, features, targets, batch: int = 8192, steps: int = 1000, lr: float = 1e-3, seed: int = 0):
        import torch

        _check(features, N_IN)
        _check(targets, N_OUT)
        losses = np.zeros(steps, np.float32)
        torch.cuda.synchronize()
        rc = native.load().cc_mlp_train(self.h, C.c_void_p(features.data_ptr()), C.c_void_p(targets.data_ptr()),
                                        features.shape[0], int(batch), int(steps), float(lr), int(seed), _fp(losses))
        if rc != 0:
            raise self._err(rc)
        return losses

    def save(self, path) -> None:
        np.savez(path, params=self.parameters())

    @classmethod
    def load(cls, path) -> "Mlp":
        m = cls(0)
        with np.load(path) as z:
            m.set_parameters(z["params"])
        return m
