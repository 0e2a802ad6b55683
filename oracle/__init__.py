"""Oracle: CPU restatement of the reference's hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``cufcm_fil_b200``) never imports it and has no CPU fallback.

Contents
  rpy_apply / mobility_*     RPY block products (C, ``rpy_oracle.c``), following
                             src/cilia/cuda_functions.cu:9-757
  beat                       prescribed Fulford-Blake beat kinematics,
                             src/cilia/filament.cpp:684-1230, 1336-1500
  implicit                   RHS, preconditioner, saddle product and GMRES,
                             src/cilia/mobility/mobility_solver.cpp:242-2669

Parity status: the implicit path is pinned against the reference's own
generalised-force tables (input/forcing/*_NSEG=20_SEP=2.600000.dat) and
arclength tables; the RPY blocks are additionally checked against the
reference's CUDA kernels compiled from its sources (oracle/_ref).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from . import build as _build

_HERE = Path(__file__).resolve().parent
_lib = None


def lib():
    """Loads (building if needed) the oracle's C library."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not path.exists():
            _build.build()
        L = ctypes.CDLL(str(path))
        for suffix, real in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            fn = getattr(L, f"oracle_rpy_apply_{suffix}")
            fn.restype = None
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int64, ctypes.c_void_p, real, ctypes.c_void_p, ctypes.c_int64,
                           ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, real, ctypes.c_int64,
                           real, ctypes.c_void_p, ctypes.c_int]
            nt = getattr(L, f"oracle_num_threads_{suffix}")
            nt.restype = ctypes.c_int
            nt.argtypes = []
        _lib = L
    return _lib


def num_threads() -> int:
    return lib().oracle_num_threads_f64()


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def rpy_apply(xt, xs, fs, *, wall, vdof, fdof, self_by_index=False, at=1.0, as_=1.0, mu=1.0,
              t_ids=None, t_off=0, s_off=0, vt=None, dtype=np.float64, nthreads=0):
    """V_t (+)= M(t <- s) F_s.

    xt [nt,3], xs [ns,3], fs [ns,fdof]; returns vt [nt,vdof] (accumulated into
    ``vt`` when given).  ``self_by_index``: in wall mode a target whose global
    id equals a source's global id uses the self block (cuda_functions.cu:24).
    """
    xt = np.ascontiguousarray(xt, dtype=dtype).reshape(-1, 3)
    xs = np.ascontiguousarray(xs, dtype=dtype).reshape(-1, 3)
    fs = np.ascontiguousarray(fs, dtype=dtype).reshape(-1, fdof)
    nt, ns = xt.shape[0], xs.shape[0]
    if vt is None:
        vt = np.zeros((nt, vdof), dtype=dtype)
    assert vt.dtype == dtype and vt.shape == (nt, vdof) and vt.flags.c_contiguous
    ids = None
    if t_ids is not None:
        ids = np.ascontiguousarray(t_ids, dtype=np.int64)
        assert ids.shape == (nt,)
    fn = lib().oracle_rpy_apply_f64 if dtype == np.float64 else lib().oracle_rpy_apply_f32
    fn(int(wall), int(vdof), int(fdof), int(bool(self_by_index)), nt, _ptr(xt), at, _ptr(ids), int(t_off),
       ns, _ptr(xs), _ptr(fs), as_, int(s_off), mu, _ptr(vt), int(nthreads))
    return vt


def mobility_full(x_segs, f_segs, x_blobs=None, f_blobs=None, *, wall, seg_dof, seg_radius=1.0,
                  blob_radius=1.0, mu=1.0, dtype=np.float64, nthreads=0, seg_targets=None):
    """Reference evaluate_full_mobility (rpy_mobility_solver.cu:330-338) in FP64.

    Host layouts as the reference: x_segs [3N], f_segs [6N] -> v_segs [6N],
    x_blobs/f_blobs [3B] -> v_blobs [3B].  ``seg_targets`` restricts the
    segment rows that are evaluated (indices; the returned v_segs then has
    those rows only).
    """
    xs = np.asarray(x_segs, dtype=dtype).reshape(-1, 3)
    fs6 = np.asarray(f_segs, dtype=dtype).reshape(-1, 6)
    ns = xs.shape[0]
    fs = fs6[:, :seg_dof]
    xb = np.zeros((0, 3), dtype) if x_blobs is None else np.asarray(x_blobs, dtype=dtype).reshape(-1, 3)
    fb = np.zeros((0, 3), dtype) if f_blobs is None else np.asarray(f_blobs, dtype=dtype).reshape(-1, 3)
    nb = xb.shape[0]
    if seg_targets is None:
        xt, ids = xs, None
    else:
        ids = np.asarray(seg_targets, dtype=np.int64)
        xt = xs[ids]
    vseg = rpy_apply(xt, xs, fs, wall=wall, vdof=seg_dof, fdof=seg_dof, self_by_index=True, at=seg_radius,
                     as_=seg_radius, mu=mu, t_ids=ids, dtype=dtype, nthreads=nthreads)
    if nb:
        rpy_apply(xt, xb, fb, wall=wall, vdof=seg_dof, fdof=3, self_by_index=False, at=seg_radius,
                  as_=blob_radius, mu=mu, vt=vseg, dtype=dtype, nthreads=nthreads)
    v_segs = np.zeros((xt.shape[0], 6), dtype=dtype)
    v_segs[:, :seg_dof] = vseg
    v_blobs = np.zeros((nb, 3), dtype=dtype)
    if nb:
        rpy_apply(xb, xb, fb, wall=wall, vdof=3, fdof=3, self_by_index=True, at=blob_radius, as_=blob_radius,
                  mu=mu, vt=v_blobs, dtype=dtype, nthreads=nthreads)
        if ns:
            rpy_apply(xb, xs, fs, wall=wall, vdof=3, fdof=seg_dof, self_by_index=False, at=blob_radius,
                      as_=seg_radius, mu=mu, vt=v_blobs, dtype=dtype, nthreads=nthreads)
    return v_segs.reshape(-1), v_blobs.reshape(-1)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
