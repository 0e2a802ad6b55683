"""Host mirror of the reference's free swimmer: one rigid spherical body carrying prescribed cilia.

``CiliatedSwimmer`` stands in for the swimmer object (a rigid_body with its
filaments) and ``mobility_solver`` that ``cilia_sim_main.cu`` drives for
CILIA_TYPE 3 with a free body (BODY_OR_SURFACE_TYPE 2, BODY_VELOCITY_TYPE 0):
one :meth:`step` is swimmer::initial_guess, mobility_solver::compute_velocities
and the explicit body update (cilia_sim_main.cu:405-416, 700-716), executed on
the device by libcufil.so (cf_swim_*).

:func:`sphere_geometry` builds the body-frame positions the reference derives
from its seeding files (swimmer.cpp:357-375, rigid_body.cpp:376-380): a sphere
of diameter ``ar`` times the filament length, blobs on its surface, filament
bases one blob radius plus half a segment spacing above it.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .sim import GmresResult


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


@dataclass
class SphereGeometry:
    fil_refs: np.ndarray    # [F, 3] filament bases in the body frame
    fil_dirs: np.ndarray    # [F, 3] outward unit normals
    blob_refs: np.ndarray   # [B, 3] blob positions in the body frame
    radius: float           # body radius


def sphere_geometry(fil_normals, blob_normals, *, ar: float, nseg: int = 20, seg_sep: float = 2.6) -> SphereGeometry:
    """Body-frame references of a sphere of diameter AXIS_DIR_BODY_LENGTH = ar * FIL_LENGTH
    (FIL_LENGTH = seg_sep * (nseg - 1), RSEG = RBLOB = 1): blobs at radius * normal, filament
    bases at (radius + RBLOB + 0.5 DL) * normal (BASE_HEIGHT_ABOVE_SURFACE = 0.5 DL)."""
    fn = np.asarray(fil_normals, np.float64).reshape(-1, 3)
    bn = np.asarray(blob_normals, np.float64).reshape(-1, 3)
    fn = fn / np.linalg.norm(fn, axis=1, keepdims=True)
    bn = bn / np.linalg.norm(bn, axis=1, keepdims=True)
    radius = 0.5 * ar * seg_sep * (nseg - 1)
    return SphereGeometry(fil_refs=(radius + 1.0 + 0.5 * seg_sep) * fn, fil_dirs=fn, blob_refs=radius * bn,
                          radius=radius)


def fibonacci_normals(n: int, offset: float = 0.5) -> np.ndarray:
    """n roughly uniform unit vectors (a Fibonacci lattice on the sphere); none lies exactly on the
    z axis, so every filament has a well-defined polar direction."""
    k = np.arange(n, dtype=np.float64) + offset
    z = 1.0 - 2.0 * k / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = np.pi * (3.0 - np.sqrt(5.0)) * k
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


class CiliatedSwimmer:
    """One free body with prescribed cilia on the device (cf_swim)."""

    def __init__(self, *, geometry: SphereGeometry, nseg=20, seg_sep=2.6, beat=_lib.CF_BEAT_FULFORD_BLAKE,
                 dt=1.0 / 300, spring_factor=0.01, gmres_tol=1e-6, gmres_max_iter=350, omega0=None, phase0=None,
                 angle0=None, phase_refs=None, angle_refs=None, s_table=None, s_tol_factor=0.0, body_x0=None,
                 body_q0=None, device=0):
        keep = []

        def arr(x, n=None):
            if x is None:
                return None
            a = np.ascontiguousarray(x, np.float64).ravel()
            if n is not None and a.size != n:
                raise ValueError(f"expected {n} values, got {a.size}")
            keep.append(a)
            return a

        F = geometry.fil_refs.shape[0]
        B = geometry.blob_refs.shape[0]
        fr, fd, br = arr(geometry.fil_refs, 3 * F), arr(geometry.fil_dirs, 3 * F), arr(geometry.blob_refs, 3 * B)
        om, ph, an = arr(omega0, F), arr(phase0, F), arr(angle0, F)
        pr, ar = arr(phase_refs), arr(angle_refs)
        bx, bq = arr(body_x0, 3), arr(body_q0, 4)
        st = None if s_table is None else np.ascontiguousarray(s_table, np.float64)
        if st is not None:
            keep.append(st)
        cfg = _lib.SwimConfig(
            n_fil=F, n_seg=int(nseg), n_blob=B, seg_sep=float(seg_sep), beat=int(beat), dt=float(dt),
            spring_factor=float(spring_factor), gmres_tol=float(gmres_tol), gmres_max_iter=int(gmres_max_iter),
            fil_refs=_p(fr), fil_dirs=_p(fd), blob_refs=_p(br), body_x0=_p(bx), body_q0=_p(bq), omega0=_p(om),
            phase0=_p(ph), angle0=_p(an), gen_phase_force_refs=_p(pr), n_gen_phase_refs=0 if pr is None else pr.size,
            gen_angle_force_refs=_p(ar), n_gen_angle_refs=0 if ar is None else ar.size, s_values_ref=_p(st),
            s_ref_rows=0 if st is None else st.shape[0], s_ref_cols=0 if st is None else st.shape[1],
            s_tol_factor=float(s_tol_factor), device=int(device))
        h = ctypes.c_void_p()
        _lib.call("cf_swim_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self.n_fil, self.n_blob, self.nseg = F, B, int(nseg)
        self.size = _lib.load().cf_swim_system_size(h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_swim_destroy", self._h)
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

    def step(self, nt: int) -> GmresResult:
        """One step; raises CufilError on a non-finite solve, returns the result otherwise
        (status CF_NOT_CONVERGED when GMRES stopped at its cap, as the reference carries on)."""
        it, rel = ctypes.c_int(), ctypes.c_double()
        rc = _lib.call("cf_swim_step", self._h, int(nt), ctypes.byref(it), ctypes.byref(rel),
                       ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED))
        return GmresResult(it.value, rel.value, rc)

    def state(self) -> dict:
        F = self.n_fil
        out = {k: np.zeros(F) for k in ("phase", "angle", "phase_dot", "angle_dot")}
        out["body_x"], out["body_q"], out["body_v"] = np.zeros(3), np.zeros(4), np.zeros(6)
        _lib.call("cf_swim_get_state", self._h, *(_p(out[k]) for k in ("phase", "angle", "phase_dot", "angle_dot",
                                                                        "body_x", "body_q", "body_v")))
        return out

    def particles(self):
        """(segment positions [N, 3], blob positions [B, 3], segment forces [N, 3], blob forces [B, 3])."""
        N, B = self.n_fil * self.nseg, self.n_blob
        xs, xb, fs, fb = np.zeros((N, 3)), np.zeros((B, 3)), np.zeros((N, 3)), np.zeros((B, 3))
        _lib.call("cf_swim_get_particles", self._h, _p(xs), _p(xb), _p(fs), _p(fb))
        return xs, xb, fs, fb

    def directions(self):
        """(vel_dir_phase [N, 3], vel_dir_angle [N, 3]) of the last step."""
        N = self.n_fil * self.nseg
        kp, ka = np.zeros((N, 3)), np.zeros((N, 3))
        _lib.call("cf_swim_get_directions", self._h, _p(kp), _p(ka))
        return kp, ka

    def tips(self) -> np.ndarray:
        xs = self.particles()[0]
        return xs.reshape(self.n_fil, self.nseg, 3)[:, -1, :]

    def system_matrix_mult_new(self, v) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64)
        out = np.zeros(self.size)
        _lib.call("cf_swim_system_matvec", self._h, _p(v), _p(out))
        return out

    def apply_preconditioner_new(self, v) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64)
        out = np.zeros(self.size)
        _lib.call("cf_swim_apply_preconditioner", self._h, _p(v), _p(out))
        return out
