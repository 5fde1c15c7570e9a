"""The proposal network over the C ABI (lenia_mlp_*): a multilayer
perceptron trained on the GPU by the library's own kernels.  Inputs and
targets are CUDA tensors (torch is used only to hold device memory)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class MLP:
    def __init__(self, n_in: int, hidden: int = 256, seed: int = 0):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        st = self._lib.lenia_mlp_create(int(n_in), int(hidden), ctypes.c_ulonglong(seed), ctypes.byref(h))
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, "lenia_mlp_create failed")
        self._h = h
        self.n_in, self.hidden = n_in, hidden

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lenia_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _lib.LENIA_OK:
            raise _lib.LeniaError(st, self._lib.lenia_mlp_last_error(self._h).decode())

    @property
    def n_params(self) -> int:
        return int(self._lib.lenia_mlp_param_count(self._h))

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        self._check(self._lib.lenia_mlp_get_params(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._lib.lenia_mlp_set_params(self._h, p.ctypes.data_as(ctypes.c_void_p), p.size))

    def grads(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        self._check(self._lib.lenia_mlp_get_grads(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def forward(self, x, stream: int = 0):
        import torch
        x = x.contiguous()
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        self._check(self._lib.lenia_mlp_forward(self._h, ctypes.c_void_p(x.data_ptr()), x.shape[0],
                                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)))
        return out

    def gradients(self, x, y, stream: int = 0) -> float:
        loss = ctypes.c_float()
        x, y = x.contiguous(), y.contiguous()
        self._check(self._lib.lenia_mlp_gradients(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                                  x.shape[0], ctypes.byref(loss), ctypes.c_void_p(stream)))
        return loss.value

    def train_step(self, x, y, lr: float = 1e-3, wd: float = 0.0, stream: int = 0) -> float:
        loss = ctypes.c_float()
        x, y = x.contiguous(), y.contiguous()
        self._check(self._lib.lenia_mlp_train_step(self._h, ctypes.c_void_p(x.data_ptr()),
                                                   ctypes.c_void_p(y.data_ptr()), x.shape[0], ctypes.c_float(lr),
                                                   ctypes.c_float(wd), ctypes.byref(loss), ctypes.c_void_p(stream)))
        return loss.value


def split_params(p: np.ndarray, dims):
    """[(W, b)] per layer from the flat layout (W out x in, then b)."""
    out, off = [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        W = p[off:off + a * b].reshape(b, a)
        off += a * b
        bias = p[off:off + b]
        off += b
        out.append((W, bias))
    return out
