"""Prescribed-beat kinematics of the reference, restated in FP64 (test infrastructure only).

Follows racksa/CUFCM_FIL src/cilia/filament.cpp:
  fill_fourier_coeff_mats     :684-960   (Fulford & Blake tables; SHAPE_SEQUENCE 1 and 4)
  fitted_shape_tangent        :962-990
  fitted_shape                :992-1024
  fitted_shape_velocity_direction :1026-1052
  fitted_curve_length         :1054-1094 (trapezoid rule, 10*NSEG intervals)
  find_fitted_shape_s         :1096-1230 (bisection in WRITE_GENERALISED_FORCES mode,
                                           bilinear table interpolation otherwise)
  initial_guess (prescribed)  :1336-1500 (positions and velocity directions)
and the wall filament frame built in filament::initial_setup (:224-430) from
the reference's quaternion helpers (src/general/quaternion.cpp:197-345).

The coefficient tables are the fitted Fourier/polynomial beat of Fulford &
Blake as tabulated by Ito, Omori & Ishikawa (2019), Table 1, in the two
scalings the reference uses; they are data and must match it value for value.
"""
from __future__ import annotations

import math

import numpy as np

# [mode, degree] layout: x(s, psi) = sum_n c_n(psi) A[n, d] s^(d+1) + sum_{n>=1} sin(n psi) B[n-1, d] s^(d+1)
FB_TABLES = {
    # SHAPE_SEQUENCE 1: scaled so that the mean curve length is 1, zero-mode pre-halved.
    1: dict(
        Ax=[[9.7204e-01, -2.8315e-01, 4.9243e-02], [-1.8466e-02, -1.2926e-01, 2.6981e-01],
            [1.6209e-01, -3.4983e-01, 1.9082e-01], [1.0259e-02, 3.5907e-02, -6.8736e-02]],
        Ay=[[-3.3547e-01, 4.0369e-01, 1.0362e-01], [4.0318e-01, -1.5553e+00, 7.3455e-01],
            [-9.9513e-02, 3.2829e-02, -1.2106e-01], [8.1046e-02, -3.0982e-01, 1.4568e-01]],
        Bx=[[1.9697e-01, -5.1193e-01, 3.4778e-01], [-5.1295e-02, 4.3396e-01, -3.3547e-01],
            [1.2311e-02, 1.4157e-01, -1.1695e-01]],
        By=[[2.9136e-01, 1.0721e+00, -1.0433e+00], [6.1554e-03, 3.2521e-01, -2.8315e-01],
            [-6.0528e-02, 2.3185e-01, -2.0108e-01]],
        c0=1.0),
    # SHAPE_SEQUENCE 4: the original coefficients, zero mode weighted by 1/2.
    4: dict(
        Ax=[[1.895, -0.552, 0.096], [-0.018, -0.126, 0.263], [0.158, -0.341, 0.186], [0.010, 0.035, -0.067]],
        Ay=[[-0.654, 0.787, 0.202], [0.393, -1.516, 0.716], [-0.097, 0.032, -0.118], [0.079, -0.302, 0.142]],
        Bx=[[0.192, -0.499, 0.339], [-0.050, 0.423, -0.327], [0.012, 0.138, -0.114]],
        By=[[0.284, 1.045, -1.017], [0.006, 0.317, -0.276], [-0.059, 0.226, -0.196]],
        c0=0.5),
}


class Beat:
    def __init__(self, shape_sequence: int, nseg: int):
        t = FB_TABLES[shape_sequence]
        self.Ax, self.Ay = np.array(t["Ax"]), np.array(t["Ay"])
        self.Bx, self.By = np.array(t["Bx"]), np.array(t["By"])
        self.c0 = t["c0"]
        self.nseg = nseg
        self.modes = self.Ax.shape[0]
        self.degrees = self.Ax.shape[1]

    def _cs(self, psi):
        n = np.arange(1, self.modes)
        cos_v = np.concatenate([[self.c0], np.cos(n * psi)])
        sin_v = np.sin(n * psi)
        return cos_v, sin_v

    def shape(self, s, psi):
        """(x, y) of fitted_shape at arclength parameter(s) s (filament.cpp:992-1024)."""
        s = np.atleast_1d(np.asarray(s, float))
        cos_v, sin_v = self._cs(psi)
        sv = s[:, None] ** (np.arange(self.degrees) + 1)[None, :]
        cx = cos_v @ self.Ax + sin_v @ self.Bx
        cy = cos_v @ self.Ay + sin_v @ self.By
        return sv @ cx, sv @ cy

    def tangent(self, s, psi):
        """d/ds of the shape (filament.cpp:962-990)."""
        s = np.atleast_1d(np.asarray(s, float))
        cos_v, sin_v = self._cs(psi)
        d = np.arange(self.degrees)
        sv = (d + 1)[None, :] * s[:, None] ** d[None, :]
        cx = cos_v @ self.Ax + sin_v @ self.Bx
        cy = cos_v @ self.Ay + sin_v @ self.By
        return sv @ cx, sv @ cy

    def velocity_direction(self, s, psi):
        """d/dpsi of the shape at fixed s (filament.cpp:1026-1052)."""
        s = np.atleast_1d(np.asarray(s, float))
        n = np.arange(1, self.modes)
        dcos = np.concatenate([[0.0], -n * np.sin(n * psi)])   # derivative of the cos row (mode 0 const)
        dsin = n * np.cos(n * psi)
        sv = s[:, None] ** (np.arange(self.degrees) + 1)[None, :]
        cx = dcos @ self.Ax + dsin @ self.Bx
        cy = dcos @ self.Ay + dsin @ self.By
        return sv @ cx, sv @ cy

    # -- arclength ------------------------------------------------------
    def _trap_table(self, psi):
        ntraps = 10 * self.nseg
        dl = 1.0 / ntraps
        grid = np.arange(ntraps + 1) * dl
        tx, ty = self.tangent(grid, psi)
        f = np.sqrt(tx * tx + ty * ty)
        cum = np.concatenate([[0.0], np.cumsum(0.5 * dl * (f[:-1] + f[1:]))])
        return dl, f, cum

    def curve_length(self, s, psi, table=None):
        """fitted_curve_length (filament.cpp:1054-1094)."""
        if s <= 0:
            return 0.0
        dl, f, cum = table if table is not None else self._trap_table(psi)
        fl = math.floor(s / dl)
        length = cum[fl]
        ce = math.ceil(s / dl)
        if ce > fl:
            length += ((s / dl - fl) / (ce - fl)) * 0.5 * dl * (f[fl] + f[ce])
        return length

    def s_bisection(self, psi, tol_factor=0.1):
        """find_fitted_shape_s in WRITE_GENERALISED_FORCES mode (filament.cpp:1128-1180).

        The bisection stops when the length fraction is within tol_factor/NSEG of its target;
        the reference code uses 0.1 (filament.cpp:1143)."""
        n = self.nseg
        table = self._trap_table(psi)
        s = np.zeros(n)
        s[-1] = 1.0
        total = self.curve_length(1.0, psi, table)
        tol = tol_factor / n
        for k in range(1, n - 1):
            target = k / (n - 1)
            lo, hi = s[k - 1], 1.0
            est = 0.5 * (lo + hi)
            frac = self.curve_length(est, psi, table) / total
            while abs(frac - target) > tol:
                if frac > target:
                    hi = est
                else:
                    lo = est
                est = 0.5 * (lo + hi)
                frac = self.curve_length(est, psi, table) / total
            s[k] = est
        return s

    def s_from_table(self, psi, table):
        """find_fitted_shape_s with a reference table (filament.cpp:1186-1224)."""
        rows, cols = table.shape
        n = self.nseg
        idx = 0.5 * psi / math.pi
        idx -= math.floor(idx)
        idx *= rows
        lo = int(idx)
        if lo == rows:
            svec = table[0]
        else:
            up = 0 if lo == rows - 1 else lo + 1
            svec = table[lo] + (table[up] - table[lo]) * (idx - lo)
        s = np.zeros(n)
        s[-1] = 1.0
        for k in range(1, n - 1):
            si = (cols - 1) * k / (n - 1)
            sl = int(si)
            s[k] = svec[sl] + (si - sl) * (svec[sl + 1] - svec[sl])
        return s


def wall_frame() -> np.ndarray:
    """Rotation R of a filament seeded on the wall with dir = e_z (filament.cpp:224-430).

    qtemp = (dir_x, 0, -dir_z, dir_y) -> sqrt_in_place_ortho -> (1/sqrt2, 0, -1/sqrt2, 0);
    the polar direction is degenerate on the wall so q2 is the identity; R = rot_mat(qtemp)
    maps the reference x axis to e_z and keeps e_y."""
    q0, q1, q2, q3 = 1.0 / math.sqrt(2.0), 0.0, -1.0 / math.sqrt(2.0), 0.0
    return quat_rot(q0, q1, q2, q3)


def quat_rot(q0, q1, q2, q3) -> np.ndarray:
    """quaternion::rot_mat (quaternion.cpp:305-345)."""
    return np.array([
        [1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
        [2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1)],
        [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)],
    ])


def filament_kinematics(beat: Beat, s, psi, angle, base, R, fil_length):
    """Segment positions and velocity directions of one filament (filament.cpp:1378-1500).

    Returns x [nseg,3], k_phase [nseg,3], k_angle [nseg,3] (segment 0 at the base, zero directions)."""
    n = beat.nseg
    ca, sa = math.cos(angle), math.sin(angle)
    Rshape = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])  # rotation about reference z
    x = np.zeros((n, 3))
    kp = np.zeros((n, 3))
    ka = np.zeros((n, 3))
    x[0] = base
    sx, sy = beat.shape(s[1:], psi)
    vx, vy = beat.velocity_direction(s[1:], psi)
    ref = fil_length * (Rshape @ np.stack([sx, sy, np.zeros_like(sx)]))       # [3, n-1]
    x[1:] = base + (R @ ref).T
    ez_cross = np.stack([-ref[1], ref[0], np.zeros_like(ref[0])])            # e_z x ref
    ka[1:] = (R @ ez_cross).T
    kp[1:] = (fil_length * (R @ Rshape @ np.stack([vx, vy, np.zeros_like(vx)]))).T
    return x, kp, ka
