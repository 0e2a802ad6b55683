"""Host mirror of the reference's cuFCM solver and its mobility adapter.

``FcmSolver`` stands in for ``FCM_solver`` (src/cufcm/CUFCM_SOLVER.cuh:5-228)
configured like its ``simulation_info`` file (N, rh, alpha, beta, eta, nx, ny,
nz, boxsize), translation only; ``hydrodynamic_solver`` applies the fast FCM
mobility to positions and forces.  ``evaluate_full_mobility`` follows
``fcm_mobility_solver::evaluate_full_mobility`` (fcm_mobility_solver.cu:463-502)
with the reference's segment/blob host layouts.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


class FcmSolver:
    def __init__(self, n, *, rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=256, ny=256, nz=256, boxsize=4000.0,
                 device=0):
        self.n = int(n)
        cfg = _lib.FcmConfig(self.n, float(rh), float(alpha), float(beta), float(eta), int(nx), int(ny), int(nz),
                             float(boxsize), int(device))
        h = ctypes.c_void_p()
        _lib.call("cf_fcm_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_fcm_destroy", self._h)
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

    def info(self) -> dict:
        out = np.zeros(9)
        _lib.call("cf_fcm_info", self._h, _p(out))
        keys = ["ngd", "dx", "sigma", "Sigma", "Rc", "Mx", "My", "Mz", "self_mobility"]
        return dict(zip(keys, out.tolist()))

    STAGES = ("clear", "hash_sort", "spread", "fft_solve", "gather", "correction")

    def set_timing(self, enable: bool = True):
        _lib.call("cf_fcm_set_timing", self._h, int(bool(enable)))

    def stage_times(self) -> dict:
        """Milliseconds of each stage of the last apply (timing must be on)."""
        out = np.zeros(6, np.float32)
        _lib.call("cf_fcm_stage_times", self._h, _p(out))
        return dict(zip(self.STAGES, out.tolist()))

    def hydrodynamic_solver(self, Y, F) -> np.ndarray:
        """V = M_FCM F for positions Y [N,3] and forces F [N,3] (host arrays)."""
        Y = np.ascontiguousarray(Y, np.float32).ravel()
        F = np.ascontiguousarray(F, np.float32).ravel()
        V = np.zeros(3 * self.n, np.float32)
        _lib.call("cf_fcm_apply", self._h, _p(Y), _p(F), _p(V))
        return V.reshape(-1, 3)

    def apply_device(self, Y, F, V, stream=None):
        """Same on device-resident torch tensors [3N] float32, ordered on `stream`."""
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.call("cf_fcm_apply_device", self._h, ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(F.data_ptr()),
                  ctypes.c_void_p(V.data_ptr()), st)

    def evaluate_full_mobility(self, x_segs, f_segs, x_blobs=None, f_blobs=None):
        """Segments then blobs in the reference host layouts; returns (v_segs [6Ns], v_blobs [3Nb])."""
        xs = np.ascontiguousarray(x_segs, np.float32).ravel()
        fs = np.ascontiguousarray(f_segs, np.float32).ravel()
        ns = xs.size // 3
        xb = np.ascontiguousarray(x_blobs if x_blobs is not None else [], np.float32).ravel()
        fb = np.ascontiguousarray(f_blobs if f_blobs is not None else [], np.float32).ravel()
        vs = np.zeros(6 * ns, np.float32)
        vb = np.zeros(xb.size, np.float32)
        _lib.call("cf_fcm_apply_segments_blobs", self._h, ns, _p(xs), _p(xb), _p(fs), _p(fb), _p(vs), _p(vb))
        return vs, vb
