"""Host side of cf_flow: the reference's flow-field post-processor (flow_field_evaluator).

Flow velocities at field points from the segment forces and torques (and blob
forces) a simulation saved; see include/cufil.h for the terms.  Arrays are in
the reference's layouts: x_flow [Nf,3], x_segs [S,3], f_segs [S,6],
x_blobs / f_blobs [B,3], x_bodies [Nbod,3].
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


class FlowFieldEvaluator:
    def __init__(self, max_flow: int, max_seg: int, max_blob: int = 0, max_bodies: int = 1, mu: float = 1.0,
                 remove_net_force: bool = False, device: int = 0):
        cfg = _lib.FlowConfig(int(max_flow), int(max_seg), int(max_blob), int(max_bodies), float(mu),
                              int(bool(remove_net_force)), int(device))
        h = ctypes.c_void_p()
        _lib.call("cf_flow_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_flow_destroy", self._h)
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

    def velocities(self, x_flow, x_segs, f_segs, *, n_seg_per_body=None, x_blobs=None, f_blobs=None,
                   n_blob_per_body=0, x_bodies=None) -> np.ndarray:
        """Flow velocities [Nf,3] (flow_field_evaluator::velocities), synchronous."""
        xf = np.ascontiguousarray(x_flow, np.float32).reshape(-1, 3)
        xs = np.ascontiguousarray(x_segs, np.float32).reshape(-1, 3)
        fs = np.ascontiguousarray(f_segs, np.float32).reshape(-1, 6)
        xb = None if x_blobs is None else np.ascontiguousarray(x_blobs, np.float32).reshape(-1, 3)
        fb = None if f_blobs is None else np.ascontiguousarray(f_blobs, np.float32).reshape(-1, 3)
        xd = None if x_bodies is None else np.ascontiguousarray(x_bodies, np.float32).reshape(-1, 3)
        nb = 0 if xb is None else xb.shape[0]
        ns_pb = xs.shape[0] if n_seg_per_body is None else int(n_seg_per_body)
        v = np.zeros_like(xf)
        _lib.call("cf_flow_velocities", self._h, _p(xf), xf.shape[0], _p(xs), _p(fs), xs.shape[0], ns_pb, _p(xb),
                  _p(fb), nb, int(n_blob_per_body), _p(xd), _p(v))
        return v
