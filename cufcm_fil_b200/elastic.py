"""Host mirror of the reference's elastic-filament path: instability-driven cilia on a wall.

``ElasticCiliaSimulation`` stands in for the swimmer/filament objects and the
``broyden_solver`` that ``cilia_sim_main.cu`` drives for CILIA_TYPE 0 on an
INFINITE_PLANE_WALL: one :meth:`step` is filament::initial_guess, the internal
forces, the 6x6 wall mobility with barrier forces, compute_errors and
Broyden's method to tolerance (cilia_sim_main.cu:405-560), executed on the
device by libcufil.so (cf_elastic_*).  Constants default to the reference's
(KB = KT = 1800, DIMENSIONLESS_FORCE = 220, TOL = 1e-4, 400 Broyden
iterations, Jacobian confidence 0.1, repulsion factor 2).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class ElasticCiliaSimulation:
    def __init__(self, *, bases, nseg=20, seg_sep=2.6, dt=36.3833 / 300, dimensionless_force=0.0, kb=0.0, kt=0.0,
                 repulsion_factor=0.0, broyden_tol=0.0, max_broyden_iter=0, jacobian_confidence=0.0, ic_type=0,
                 perturbations=None, device=0):
        self.bases = np.ascontiguousarray(bases, np.float64).reshape(-1, 3)
        self.n_fil, self.nseg = self.bases.shape[0], int(nseg)
        self._pert = None if perturbations is None else np.ascontiguousarray(perturbations, np.float64).reshape(-1)
        cfg = _lib.ElasticConfig(
            n_fil=self.n_fil, n_seg=self.nseg, seg_sep=float(seg_sep), base_pos=_p(self.bases), dt=float(dt),
            dimensionless_force=float(dimensionless_force), kb=float(kb), kt=float(kt),
            repulsion_factor=float(repulsion_factor), broyden_tol=float(broyden_tol),
            max_broyden_iter=int(max_broyden_iter), jacobian_confidence=float(jacobian_confidence),
            ic_type=int(ic_type), perturbations=_p(self._pert), device=int(device))
        h = ctypes.c_void_p()
        _lib.call("cf_elastic_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self.size = _lib.load().cf_elastic_system_size(h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_elastic_destroy", self._h)
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

    def step(self, nt: int) -> int:
        """One step; returns the Broyden iterations it took (CufilError when it did not converge)."""
        it = ctypes.c_int()
        _lib.call("cf_elastic_step", self._h, int(nt), ctypes.byref(it))
        return it.value

    def segments(self):
        """(positions [N, 3], orientations [N, 4], internal forces and torques [N, 6]), FP64."""
        N = self.n_fil * self.nseg
        x, q, f = np.zeros((N, 3)), np.zeros((N, 4)), np.zeros((N, 6))
        _lib.call("cf_elastic_get_segments", self._h, _p(x), _p(q), _p(f))
        return x, q, f

    def tips(self) -> np.ndarray:
        return self.segments()[0].reshape(self.n_fil, self.nseg, 3)[:, -1]

    def jacobian_inverse(self, m: int = 0) -> np.ndarray:
        n = 6 * self.nseg
        out = np.zeros((n, n))
        _lib.call("cf_elastic_get_jacobian_inverse", self._h, int(m), _p(out))
        return out

    def first_evaluation(self, nt: int = 0) -> np.ndarray:
        err = np.zeros(self.size)
        _lib.call("cf_elastic_first_evaluation", self._h, int(nt), _p(err))
        return err

    def stats(self) -> dict:
        last, mx, steps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        total = ctypes.c_longlong()
        _lib.call("cf_elastic_stats", self._h, ctypes.byref(last), ctypes.byref(mx), ctypes.byref(total),
                  ctypes.byref(steps))
        return dict(last=last.value, max=mx.value, total=total.value, steps=steps.value)
