"""Host side of cf_mlp: the per-filament network of the learned preconditioner.

The network (in -> H -> H -> out, ReLU) is trained and evaluated by the
library's own kernels (BF16 tensor-core GEMMs with FP32 accumulation, FP32
Adam); tensors are torch CUDA tensors (float32, contiguous, row-major).
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class FilamentMLP:
    def __init__(self, n_in: int, hidden: int = 256, n_out: int = 62, max_batch: int = 8192, seed: int = 0,
                 device: int = 0, _handle=None):
        self.n_in, self.hidden, self.n_out, self.max_batch = int(n_in), int(hidden), int(n_out), int(max_batch)
        if _handle is None:
            h = ctypes.c_void_p()
            _lib.call("cf_mlp_create", self.n_in, self.hidden, self.n_out, self.max_batch, ctypes.c_ulonglong(seed),
                      int(device), ctypes.byref(h))
        else:
            h = _handle
        self._h = h
        self.num_params = int(_lib.load().cf_mlp_num_params(h))

    def save(self, path, weight: float = 1.0) -> None:
        """Versioned checkpoint of the parameters and the correction weight (cf_precond_save)."""
        _lib.call("cf_precond_save", self._h, float(weight), str(path).encode())

    @classmethod
    def load(cls, path, max_batch: int = 8192, device: int = 0):
        """(network, weight) from a cf_precond_save checkpoint (cf_precond_load validates the file)."""
        h = ctypes.c_void_p()
        w = ctypes.c_double()
        _lib.call("cf_precond_load", str(path).encode(), int(max_batch), int(device), ctypes.byref(h), ctypes.byref(w))
        with open(path, "rb") as f:  # widths from the header the library just accepted
            n_in, hidden, n_out = struct.unpack_from("<3i", f.read(56), 16)
        return cls(n_in, hidden, n_out, max_batch, device=device, _handle=h), w.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_mlp_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def forward(self, x, y, stream=None):
        """y[n, out] = net(x[n, in]) on the device (ordered on `stream`, default the network's own)."""
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.call("cf_mlp_forward", self._h, _ptr(x), int(x.shape[0]), _ptr(y), st)

    def gradients(self, x, t):
        """(loss, flat gradient as numpy float32) of the mean squared error on one batch."""
        g = np.zeros(self.num_params, np.float32)
        loss = ctypes.c_double()
        _lib.call("cf_mlp_gradients", self._h, _ptr(x), _ptr(t), int(x.shape[0]), ctypes.c_void_p(g.ctypes.data),
                  ctypes.byref(loss))
        return loss.value, g

    def train_step(self, x, t, lr: float = 1e-3, want_loss: bool = False):
        loss = ctypes.c_double()
        _lib.call("cf_mlp_train_step", self._h, _ptr(x), _ptr(t), int(x.shape[0]), ctypes.c_float(lr),
                  ctypes.byref(loss) if want_loss else None)
        return loss.value if want_loss else None

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        _lib.call("cf_mlp_get_params", self._h, ctypes.c_void_p(p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params
        _lib.call("cf_mlp_set_params", self._h, ctypes.c_void_p(p.ctypes.data))
