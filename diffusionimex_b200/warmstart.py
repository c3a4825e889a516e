"""Learned warm start for the implicit-pressure Newton (no counterpart in the reference).

`MLP` wraps the tensor-core network of libspb6g (spb6g_mlp_*): 64 BF16 inputs
per row (the solver's features use 63), three hidden layers of 64 with SiLU, one output;
FP32 master weights trained with Adam on the device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .solver import SolverError, library

F = 64


class MLP:
    def __init__(self, device: int = 0):
        self._lib = library()
        self._h = ctypes.c_void_p()
        rc = self._lib.spb6g_mlp_create(device, ctypes.byref(self._h))
        if rc != 0:
            raise SolverError(rc, "spb6g_mlp_create")
        self.nparam = self._lib.spb6g_mlp_param_count()

    def close(self):
        if self._h:
            self._lib.spb6g_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparam
        self._check(self._lib.spb6g_mlp_set_params(self._h, p.ctypes.data), "set_params")

    def params(self) -> np.ndarray:
        p = np.empty(self.nparam, dtype=np.float32)
        self._check(self._lib.spb6g_mlp_get_params(self._h, p.ctypes.data), "get_params")
        return p

    def forward(self, X, y=None, stream=None):
        """X: (n, 64) torch.bfloat16 on the device; returns (n,) torch.float32.  stream: a
        torch.cuda.Stream to launch on without synchronising (None: synchronised call)."""
        import torch

        n = X.shape[0]
        assert X.dtype == torch.bfloat16 and X.is_contiguous() and X.shape[1] == F
        if y is None:
            y = torch.empty(n, dtype=torch.float32, device=X.device)
        if stream is None:
            torch.cuda.current_stream(X.device).synchronize()  # X complete before the handle's stream reads it
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        self._check(self._lib.spb6g_mlp_forward(self._h, X.data_ptr(), n, y.data_ptr(), st), "forward")
        return y

    def train_step(self, X, t, lr: float, want_grad: bool = False):
        """One pass over the rows: loss (and gradient); with lr > 0 one Adam step."""
        import torch

        n = X.shape[0]
        assert X.dtype == torch.bfloat16 and X.is_contiguous() and X.shape[1] == F and t.is_contiguous()
        torch.cuda.current_stream(X.device).synchronize()  # the batch complete before the handle's stream reads it
        loss = ctypes.c_float()
        g = np.empty(self.nparam, dtype=np.float32) if want_grad else None
        self._check(self._lib.spb6g_mlp_train_step(self._h, X.data_ptr(), t.data_ptr(), n, ctypes.c_float(lr),
                                                   ctypes.byref(loss), g.ctypes.data if want_grad else None),
                    "train_step")
        return (loss.value, g) if want_grad else loss.value

    def train_async(self, X, t, lr: float, stream):
        """One training pass launched on `stream` (a torch.cuda.Stream), nothing read back."""
        import torch

        assert X.dtype == torch.bfloat16 and X.is_contiguous() and X.shape[1] == F and t.is_contiguous()
        self._check(self._lib.spb6g_mlp_train_async(self._h, X.data_ptr(), t.data_ptr(), X.shape[0], ctypes.c_float(lr),
                                                    ctypes.c_void_p(stream.cuda_stream)), "train_async")

    def last_loss(self, stream=None) -> float:
        """Sum of squared errors of the last pass (waits for `stream`)."""
        loss = ctypes.c_float()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        self._check(self._lib.spb6g_mlp_last_loss(self._h, st, ctypes.byref(loss)), "last_loss")
        return loss.value

    @staticmethod
    def _check(rc, what):
        if rc != 0:
            raise SolverError(rc, what)
