"""Fourier-neural-operator surrogate: handle over ``fi_fno_*`` (include/fastiso_b200.h).

``FNO`` owns a network on one GPU; every tensor argument is a contiguous float32 CUDA
tensor (the C ABI takes its device pointer).  Input x is [B, 6, S, S] and output y is
[B, S, S], x fastest in both (``a[b, c, j, i]`` is cell (x_i, y_j)).  The forward pass,
the backward pass and Adam run in libfastiso_b200.so on the tensor cores; nothing here
computes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

N_IN = 6


class FNO:
    """A surrogate network of grid size S, training batches up to ``max_batch``."""

    def __init__(self, S: int = 128, max_batch: int = 32, device: int = 0, seed: int = 0):
        self._lib = abi.load_library()
        self.S, self.max_batch, self.device = int(S), int(max_batch), int(device)
        h = C.c_void_p()
        rc = self._lib.fi_fno_create(self.S, self.max_batch, self.device, C.c_uint64(seed), C.byref(h))
        if rc != 0:
            raise abi.FiError(rc, f"fi_fno_create(S={S}, max_batch={max_batch}) failed")
        self._h = h
        self.n_params = int(self._lib.fi_fno_num_params(h))

    # -- lifecycle -------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.fi_fno_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = self._lib.fi_fno_last_error(self._h)
            raise abi.FiError(rc, f"{what}: {msg.decode() if msg else ''}")

    # -- parameters ------------------------------------------------------------------
    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.fi_fno_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size),
                    "fi_fno_get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        self._check(self._lib.fi_fno_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size),
                    "fi_fno_set_params")

    def get_grads(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.fi_fno_get_grads(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size),
                    "fi_fno_get_grads")
        return out

    # -- compute ---------------------------------------------------------------------
    def _tensor(self, t, shape, name):
        import torch

        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise TypeError(f"{name} must be a contiguous float32 CUDA tensor")
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
        return C.c_void_p(t.data_ptr())

    @staticmethod
    def _sync_producer():
        # the library's stream orders after the legacy default stream; work queued on
        # another torch stream must be finished first
        import torch

        if torch.cuda.current_stream() != torch.cuda.default_stream():
            torch.cuda.current_stream().synchronize()

    def forward(self, x, out=None):
        """y = FNO(x) for one batch of at most max_batch samples."""
        import torch

        B = x.shape[0]
        xp = self._tensor(x, (B, N_IN, self.S, self.S), "x")
        y = out if out is not None else torch.empty((B, self.S, self.S), dtype=torch.float32, device=x.device)
        yp = self._tensor(y, (B, self.S, self.S), "y")
        self._sync_producer()
        self._check(self._lib.fi_fno_forward(self._h, B, xp, yp), "fi_fno_forward")
        return y

    def predict(self, x):
        """Forward pass over any number of samples, in chunks of max_batch."""
        import torch

        y = torch.empty((x.shape[0], self.S, self.S), dtype=torch.float32, device=x.device)
        for i in range(0, x.shape[0], self.max_batch):
            self.forward(x[i:i + self.max_batch].contiguous(), out=y[i:i + self.max_batch])
        return y

    def backward(self, dy) -> None:
        """Gradients of sum(dy * y) for the last forward pass (read with get_grads)."""
        B = dy.shape[0]
        dp = self._tensor(dy, (B, self.S, self.S), "dy")
        self._sync_producer()
        self._check(self._lib.fi_fno_backward(self._h, B, dp), "fi_fno_backward")

    def train_step(self, x, target, lr: float, weights=None) -> float:
        """Forward, mean-squared-error loss (per-sample weights [B] if given), backward and
        one Adam step; returns the loss."""
        B = x.shape[0]
        xp = self._tensor(x, (B, N_IN, self.S, self.S), "x")
        tp = self._tensor(target, (B, self.S, self.S), "target")
        wp = None if weights is None else self._tensor(weights, (B,), "weights")
        loss = C.c_float(0.0)
        self._sync_producer()
        self._check(self._lib.fi_fno_train_step_weighted(self._h, B, xp, tp, wp, C.c_float(lr), C.byref(loss)),
                    "fi_fno_train_step")
        return float(loss.value)

    def loss_backward(self, x, target, weights=None) -> float:
        """Forward, loss and backward without the optimizer step (data-parallel training:
        reduce ``grads_tensor()`` across ranks, then ``adam``)."""
        B = x.shape[0]
        xp = self._tensor(x, (B, N_IN, self.S, self.S), "x")
        tp = self._tensor(target, (B, self.S, self.S), "target")
        wp = None if weights is None else self._tensor(weights, (B,), "weights")
        loss = C.c_float(0.0)
        self._sync_producer()
        self._check(self._lib.fi_fno_loss_backward(self._h, B, xp, tp, wp, C.byref(loss)), "fi_fno_loss_backward")
        return float(loss.value)

    def grads_tensor(self):
        """The gradient vector in device memory as a float32 torch tensor (no copy; valid
        while this handle is open, rewritten by the next backward pass)."""
        import torch

        ptr = self._lib.fi_fno_grads_device(self._h)
        if not ptr:
            raise abi.FiError(abi.FI_ERR_ARG, "no gradient buffer")

        class _View:
            __cuda_array_interface__ = {"shape": (self.n_params,), "typestr": "<f4", "data": (int(ptr), False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_View(), device=f"cuda:{self.device}")

    def adam(self, lr: float) -> None:
        self._check(self._lib.fi_fno_adam(self._h, C.c_float(lr)), "fi_fno_adam")

    def set_adam(self, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
        self._check(self._lib.fi_fno_set_adam(self._h, beta1, beta2, eps), "fi_fno_set_adam")
