"""Oracle: the free swimmer's saddle product and preconditioner in FP64 -- TEST INFRASTRUCTURE ONLY.

CPU restatement (numpy) of the body branches of the reference's
mobility_solver for prescribed cilia on one free rigid body
(BODY_VELOCITY_TYPE 0, unbounded fluid, dynamic phase and shape-rotation angle):

  matvec    mobility_solver::system_matrix_mult_new, src/cilia/mobility/mobility_solver.cpp:1887-2105
  precond   mobility_solver::apply_preconditioner_new, mobility_solver.cpp:1244-1475, with the body's
            6x6 matrix of swimmer::make_precon_mat, src/cilia/swimmer.cpp:1175-1349
  schur     that 6x6 matrix before its inversion

Saddle layout [3N segment forces | 3B blob forces | V, Omega | F phase rates | F angle rates] with
N = F * nseg; all radii 1, MU = 1, so both segment and blob mobility factors are 6 pi.
The geometry (segment and blob positions, body centre, velocity directions) is an input: the
trajectory is pinned separately against the reference's own step code (ref_step.run_body).
"""
from __future__ import annotations

import numpy as np

from . import rpy_apply

MOB = 6.0 * np.pi  # seg_mob_inv = blob_mob_inv = 6 pi MU R with R = MU = 1


def _rcross(d):
    """rcross(d) of src/general/matrix.cpp:665-679 (rcross(d) w = w x d)."""
    return np.array([[0.0, d[2], -d[1]], [-d[2], 0.0, d[0]], [d[1], -d[0], 0.0]])


def _split(v, N, B, F):
    v = np.asarray(v, np.float64)
    fs = v[:3 * N].reshape(N, 3)
    fb = v[3 * N:3 * (N + B)].reshape(B, 3)
    o = 3 * (N + B)
    return fs, fb, v[o:o + 3], v[o + 3:o + 6], v[o + 6:o + 6 + F], v[o + 6 + F:o + 6 + 2 * F]


def matvec(xs, xb, body_x, kp, ka, v, nseg):
    """A v for the swimmer's saddle system (mobility_solver.cpp:1887-2105)."""
    xs = np.asarray(xs, np.float64).reshape(-1, 3)
    xb = np.asarray(xb, np.float64).reshape(-1, 3)
    kp = np.asarray(kp, np.float64).reshape(-1, 3)
    ka = np.asarray(ka, np.float64).reshape(-1, 3)
    N, B = xs.shape[0], xb.shape[0]
    F = N // nseg
    fs, fb, V, W, ph, an = _split(v, N, B, F)
    xa = np.concatenate([xs, xb])
    u = rpy_apply(xa, xa, np.concatenate([fs, fb]), wall=False, vdof=3, fdof=3)
    ds = xs - body_x
    db = xb - body_x
    out = np.zeros_like(np.asarray(v, np.float64))
    rate = np.repeat(ph, nseg)[:, None] * kp + np.repeat(an, nseg)[:, None] * ka
    out[:3 * N] = (u[:N] - V - np.cross(W, ds) - rate).ravel()
    out[3 * N:3 * (N + B)] = (u[N:] - V - np.cross(W, db)).ravel()
    o = 3 * (N + B)
    out[o:o + 3] = -(fs.sum(0) + fb.sum(0))
    out[o + 3:o + 6] = -(np.cross(ds, fs).sum(0) + np.cross(db, fb).sum(0))
    out[o + 6:o + 6 + F] = -(kp * fs).reshape(F, -1).sum(1)
    out[o + 6 + F:o + 6 + 2 * F] = -(ka * fs).reshape(F, -1).sum(1)
    return out


def _filament_sums(xs, body_x, kp, ka, nseg):
    ds = (xs - body_x).reshape(-1, nseg, 3)
    kpf, kaf = kp.reshape(-1, nseg, 3), ka.reshape(-1, nseg, 3)
    vp, vt = kpf.sum(1), kaf.sum(1)
    up, ut = np.cross(ds, kpf).sum(1), np.cross(ds, kaf).sum(1)
    c11, c22, c12 = (kpf * kpf).sum((1, 2)), (kaf * kaf).sum((1, 2)), (kpf * kaf).sum((1, 2))
    det = c11 * c22 - c12 * c12
    return vp, vt, up, ut, c22 / det, c11 / det, -c12 / det


def schur(xs, xb, body_x, kp, ka, nseg):
    """KTMinvK before its inversion (swimmer::make_precon_mat, dynamic phase and angle)."""
    xs = np.asarray(xs, np.float64).reshape(-1, 3)
    xb = np.asarray(xb, np.float64).reshape(-1, 3)
    kp = np.asarray(kp, np.float64).reshape(-1, 3)
    ka = np.asarray(ka, np.float64).reshape(-1, 3)
    K = np.zeros((6, 6))
    K[:3, :3] = np.eye(3) * (xs.shape[0] + xb.shape[0]) * MOB
    for d in np.concatenate([xs - body_x, xb - body_x]):
        rc = _rcross(d)
        K[:3, 3:] += MOB * rc
        K[3:, 3:] -= MOB * rc @ rc
    K[3:, :3] = -K[:3, 3:]
    vp, vt, up, ut, i11, i22, i12 = _filament_sums(xs, body_x, kp, ka, nseg)
    C = np.zeros((6, 6))
    for m in range(vp.shape[0]):
        o = np.outer
        C[:3, :3] += o(vp[m], vp[m]) * i11[m] + o(vp[m], vt[m]) * i12[m] + o(vt[m], vp[m]) * i12[m] + \
            o(vt[m], vt[m]) * i22[m]
        C[3:, :3] += o(up[m], vp[m]) * i11[m] + o(up[m], vt[m]) * i12[m] + o(ut[m], vp[m]) * i12[m] + \
            o(ut[m], vt[m]) * i22[m]
        C[3:, 3:] += o(up[m], up[m]) * i11[m] + o(up[m], ut[m]) * i12[m] + o(ut[m], up[m]) * i12[m] + \
            o(ut[m], ut[m]) * i22[m]
    C[:3, 3:] = C[3:, :3].T
    return K - MOB * C


def precond(xs, xb, body_x, kp, ka, r, nseg):
    """P r (apply_preconditioner_new, body branch, mobility_solver.cpp:1244-1475)."""
    xs = np.asarray(xs, np.float64).reshape(-1, 3)
    xb = np.asarray(xb, np.float64).reshape(-1, 3)
    kp = np.asarray(kp, np.float64).reshape(-1, 3)
    ka = np.asarray(ka, np.float64).reshape(-1, 3)
    N, B = xs.shape[0], xb.shape[0]
    F = N // nseg
    rs, rb, rV, rW, rph, ran = _split(r, N, B, F)
    ds, db = xs - body_x, xb - body_x
    ss, sb = MOB * rs, MOB * rb                       # M^-1 r_1
    body = -np.concatenate([rV, rW])                  # -r_2
    body[:3] -= ss.sum(0) + sb.sum(0)                 # - K^T M^-1 r_1
    body[3:] -= np.cross(ds, ss).sum(0) + np.cross(db, sb).sum(0)
    vp, vt, up, ut, i11, i22, i12 = _filament_sums(xs, body_x, kp, ka, nseg)
    ph = -rph - (kp * ss).reshape(F, -1).sum(1)
    an = -ran - (ka * ss).reshape(F, -1).sum(1)
    ph, an = i11 * ph + i12 * an, i12 * ph + i22 * an  # C^-1
    body[:3] -= (ph[:, None] * vp + an[:, None] * vt).sum(0)
    body[3:] -= (ph[:, None] * up + an[:, None] * ut).sum(0)
    body = np.linalg.solve(schur(xs, xb, body_x, kp, ka, nseg), body)
    V, W = body[:3], body[3:]
    ph, an = ph / MOB, an / MOB
    ph, an = (ph - (i11 * (vp @ V) + i12 * (vt @ V) + i11 * (up @ W) + i12 * (ut @ W)),
              an - (i12 * (vp @ V) + i22 * (vt @ V) + i12 * (up @ W) + i22 * (ut @ W)))
    ss = ss + MOB * (V + np.cross(W, ds) + np.repeat(ph, nseg)[:, None] * kp + np.repeat(an, nseg)[:, None] * ka)
    sb = sb + MOB * (V + np.cross(W, db))
    return np.concatenate([ss.ravel(), sb.ravel(), V, W, ph, an])


# ---------------------------------------------------------------- whole steps
def qmul(a, b):
    """Hamilton product, scalar first (quaternion.cpp:104-118)."""
    s = a[0] * b[0] - a[1:] @ b[1:]
    v = a[0] * b[1:] + b[0] * a[1:] + np.cross(a[1:], b[1:])
    return np.concatenate([[s], v])


def _sqrt_ortho(q):
    """sqrt_in_place_ortho (quaternion.cpp:197-223) with its guard near -1."""
    q = np.array(q, np.float64)
    if q[0] < -0.999999:
        q[0] = np.sqrt(0.5 * (1.0 - 0.9999999))
        q[1:] /= 2.0 * q[0]
        nrm = np.linalg.norm(q)
        q[0] *= nrm
        q[1:] /= nrm
    else:
        q[0] = np.sqrt(0.5 * (1.0 + q[0]))
        q[1:] /= 2.0 * q[0]
    return q / np.linalg.norm(q)


def _normal(q):
    """quaternion::normal (quaternion.cpp:271-277): the image of the reference y axis."""
    s, x, y, z = q
    return np.array([2.0 * (x * y - s * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z + s * x)])


def lie_exp(u):
    """lie_exp (quaternion.cpp:500-523): identity below a rotation of 1e-6."""
    th = np.linalg.norm(u)
    if th < 1e-6:
        return np.array([1.0, 0.0, 0.0, 0.0])
    return np.concatenate([[np.cos(0.5 * th)], np.sin(0.5 * th) / th * np.asarray(u, np.float64)])


def filament_frame(direction):
    """Frame of a filament whose base direction is `direction` (filament.cpp:224-236, 368-430, no tilt):
    qtemp takes the reference x axis to the direction, q2 then turns the reference y axis onto the polar
    direction (-e_z projected off the direction); q = q2 qtemp."""
    d = np.asarray(direction, np.float64)
    d = d / np.linalg.norm(d)
    qt = _sqrt_ortho([d[0], 0.0, -d[2], d[1]])
    bn = _normal(qt)
    pol = np.array([0.0, 0.0, -1.0])
    pol = pol - (d @ pol) * d
    npol = np.linalg.norm(pol)
    if npol == 0.0:
        return qt
    pol /= npol
    q2 = _sqrt_ortho(np.concatenate([[pol @ bn], np.cross(bn, pol)]))
    return qmul(q2, qt)


class Swimmer:
    """One free body with prescribed cilia stepped on the CPU in FP64 (the oracle of cf_swim).

    Per step nt (cilia_sim_main.cu:405-416, 700-716): filament frames q_body q_ref and bases
    x_body + R_body fil_ref (swimmer::initial_guess, swimmer.cpp:433-466; filament.cpp:653-666,
    1360-1376), phase and angle advanced with the last rates when nt > 0, the beat kinematics,
    the RHS (-q_phase, -q_angle rows), GMRES on matvec with precond, then x += dt V,
    q = lie_exp(dt Omega) q."""

    def __init__(self, *, fil_refs, fil_dirs, blob_refs, nseg, seg_sep, dt, phase0, angle0, phase_refs,
                 angle_refs, s_table, spring_factor=0.01, omega0=None, tol=1e-6, max_iter=350):
        from .beat import Beat
        self.fil_refs = np.asarray(fil_refs, np.float64).reshape(-1, 3)
        self.blob_refs = np.asarray(blob_refs, np.float64).reshape(-1, 3)
        self.F, self.B, self.nseg = self.fil_refs.shape[0], self.blob_refs.shape[0], int(nseg)
        self.N = self.F * self.nseg
        self.qref = [filament_frame(d) for d in np.asarray(fil_dirs, np.float64).reshape(-1, 3)]
        self.beat = Beat(1, self.nseg)
        self.fil_length = seg_sep * (self.nseg - 1)
        self.dt, self.tol, self.max_iter = float(dt), float(tol), int(max_iter)
        self.phase = np.array(phase0, np.float64)
        self.angle = np.array(angle0, np.float64)
        self.omega0 = np.full(self.F, 2 * np.pi) if omega0 is None else np.array(omega0, np.float64)
        self.phase_dot = self.omega0.copy()
        self.angle_dot = np.zeros(self.F)
        self.phase_refs, self.angle_refs = np.asarray(phase_refs), np.asarray(angle_refs)
        self.s_table, self.spring = np.asarray(s_table), float(spring_factor)
        self.body_x, self.body_q, self.body_v = np.zeros(3), np.array([1.0, 0.0, 0.0, 0.0]), np.zeros(6)
        self.size = 3 * (self.N + self.B) + 6 + 2 * self.F
        self.sol = np.zeros(self.size)

    def geometry(self, nt):
        from .beat import filament_kinematics, quat_rot
        if nt > 0:
            self.phase = self.phase + self.phase_dot * self.dt
            self.angle = self.angle + self.angle_dot * self.dt
        Rb = quat_rot(*self.body_q)
        self.xs, self.kp, self.ka = (np.zeros((self.N, 3)) for _ in range(3))
        for m in range(self.F):
            R = quat_rot(*qmul(self.body_q, self.qref[m]))
            base = self.body_x + Rb @ self.fil_refs[m]
            s = self.beat.s_from_table(self.phase[m], self.s_table)
            sl = slice(m * self.nseg, (m + 1) * self.nseg)
            self.xs[sl], self.kp[sl], self.ka[sl] = filament_kinematics(self.beat, s, self.phase[m], self.angle[m],
                                                                        base, R, self.fil_length)
        self.xb = self.body_x + self.blob_refs @ Rb.T

    def rhs(self):
        from .implicit import cyclic_cubic_spline
        r = np.zeros(self.size)
        o = 3 * (self.N + self.B) + 6
        L3 = self.fil_length ** 3
        for m in range(self.F):
            w0 = 0.5 * self.omega0[m] / np.pi
            qa = cyclic_cubic_spline(self.phase[m], self.angle_refs) * w0
            qa -= self.spring * self.omega0[m] * L3 * self.angle[m]
            r[o + m] = -cyclic_cubic_spline(self.phase[m], self.phase_refs) * w0
            r[o + self.F + m] = -qa
        return r

    def matvec(self, v):
        return matvec(self.xs, self.xb, self.body_x, self.kp, self.ka, v, self.nseg)

    def precond(self, v):
        return precond(self.xs, self.xb, self.body_x, self.kp, self.ka, v, self.nseg)

    def step(self, nt):
        from .implicit import gmres_right
        self.geometry(nt)
        self.sol, it, rel = gmres_right(self.matvec, self.precond, self.rhs(), self.sol, self.tol,
                                        min(self.size, self.max_iter))
        o = 3 * (self.N + self.B)
        self.body_v = self.sol[o:o + 6].copy()
        self.phase_dot = self.sol[o + 6:o + 6 + self.F].copy()
        self.angle_dot = self.sol[o + 6 + self.F:].copy()
        self.body_x = self.body_x + self.dt * self.body_v[:3]
        self.body_q = qmul(lie_exp(self.dt * self.body_v[3:]), self.body_q)
        return it, rel

    def tips(self):
        return self.xs.reshape(self.F, self.nseg, 3)[:, -1]
