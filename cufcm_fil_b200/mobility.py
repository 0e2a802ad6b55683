"""Host-side mirror of the reference's RPY mobility back-end.

``RpyMobilitySolver`` follows ``rpy_mobility_solver``
(src/cilia/mobility/rpy_mobility_solver.hpp:15-64): it owns host buffers with
the same names and layouts (``x_segs_host`` [3N], ``f_segs_host`` [6N],
``v_segs_host`` [6N], ``x_blobs_host`` / ``f_blobs_host`` / ``v_blobs_host``
[3B]) and exposes the same staging / evaluation methods, each a call into
libcufil.so.  Physics objects write positions and forces into the host
buffers, exactly as the reference's filaments write through raw pointers
(mobility_solver.hpp:53-63).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


class RpyMobilitySolver:
    """RPY grand-mobility products on one B200 (wall-bounded or unbounded)."""

    def __init__(self, n_seg: int, n_blob: int = 0, *, wall: bool = True, seg_dof: int = 3,
                 seg_radius: float = 1.0, blob_radius: float = 1.0, mu: float = 1.0, device: int = 0):
        self.n_seg, self.n_blob, self.seg_dof = int(n_seg), int(n_blob), int(seg_dof)
        cfg = _lib.MobilityConfig(self.n_seg, self.n_blob, int(bool(wall)), self.seg_dof, float(seg_radius),
                                  float(blob_radius), float(mu), int(device))
        h = ctypes.c_void_p()
        _lib.call("cf_mobility_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        # allocate_host_memory (rpy_mobility_solver.cu:54-89): same buffers and layouts
        self.x_segs_host = np.zeros(3 * self.n_seg, np.float32)
        self.f_segs_host = np.zeros(6 * self.n_seg, np.float32)
        self.v_segs_host = np.zeros(6 * self.n_seg, np.float32)
        self.x_blobs_host = np.zeros(3 * self.n_blob, np.float32)
        self.f_blobs_host = np.zeros(3 * self.n_blob, np.float32)
        self.v_blobs_host = np.zeros(3 * self.n_blob, np.float32)

    # -- lifetime ---------------------------------------------------------
    def finalise(self):
        if getattr(self, "_h", None):
            _lib.call("cf_mobility_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.finalise()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.finalise()

    # -- staging (rpy_mobility_solver.cu:119-205) --------------------------
    def copy_segment_positions_to_device(self):
        _lib.call("cf_copy_segment_positions_to_device", self._h, _ptr(self.x_segs_host))

    def copy_segment_forces_to_device(self):
        _lib.call("cf_copy_segment_forces_to_device", self._h, _ptr(self.f_segs_host))

    def copy_blob_positions_to_device(self):
        _lib.call("cf_copy_blob_positions_to_device", self._h, _ptr(self.x_blobs_host))

    def copy_blob_forces_to_device(self):
        _lib.call("cf_copy_blob_forces_to_device", self._h, _ptr(self.f_blobs_host))

    def copy_segment_velocities_to_host(self):
        _lib.call("cf_copy_segment_velocities_to_host", self._h, _ptr(self.v_segs_host))

    def copy_blob_velocities_to_host(self):
        _lib.call("cf_copy_blob_velocities_to_host", self._h, _ptr(self.v_blobs_host))

    def wait_for_device(self):
        _lib.call("cf_wait_for_device", self._h)

    # -- products (rpy_mobility_solver.cu:258-338) ------------------------
    def evaluate_segment_segment_mobility(self):
        _lib.call("cf_evaluate_segment_segment_mobility", self._h)

    def evaluate_segment_blob_mobility(self):
        _lib.call("cf_evaluate_segment_blob_mobility", self._h)

    def evaluate_blob_blob_mobility(self):
        _lib.call("cf_evaluate_blob_blob_mobility", self._h)

    def evaluate_blob_segment_mobility(self):
        _lib.call("cf_evaluate_blob_segment_mobility", self._h)

    def evaluate_full_mobility(self):
        _lib.call("cf_evaluate_full_mobility", self._h)

    # -- convenience ------------------------------------------------------
    def apply(self, x_segs, f_segs, x_blobs=None, f_blobs=None):
        """One synchronous full product; returns (v_segs [6N], v_blobs [3B])."""
        self.x_segs_host[:] = np.asarray(x_segs, np.float32).ravel()
        self.f_segs_host[:] = np.asarray(f_segs, np.float32).ravel()
        if self.n_blob:
            self.x_blobs_host[:] = np.asarray(x_blobs, np.float32).ravel()
            self.f_blobs_host[:] = np.asarray(f_blobs, np.float32).ravel()
        _lib.call("cf_apply_mobility", self._h, _ptr(self.x_segs_host), _ptr(self.x_blobs_host),
                  _ptr(self.f_segs_host), _ptr(self.f_blobs_host), _ptr(self.v_segs_host), _ptr(self.v_blobs_host))
        return self.v_segs_host.copy(), self.v_blobs_host.copy()

    def apply_device(self, x_segs, f_segs, v_segs, x_blobs=None, f_blobs=None, v_blobs=None, stream=None):
        """Full product on device-resident torch tensors (AoS float32 layouts), async on `stream`."""
        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None  # None: legacy default stream
        _lib.call("cf_apply_mobility_device", self._h, p(x_segs), p(x_blobs), p(f_segs), p(f_blobs), p(v_segs),
                  p(v_blobs), st)
