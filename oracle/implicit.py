"""Implicit prescribed-cilia step of the reference, restated in FP64 (test infrastructure only).

Follows racksa/CUFCM_FIL src/cilia/mobility/mobility_solver.cpp:
  cyclic_cubic_spline_interpolation  :242-282
  assemble_rhs (PRESCRIBED_CILIA, wall)              :284-420
  apply_preconditioner_new (PRESCRIBED_BODY_VELOCITIES) :1102-1243
  system_matrix_mult_new (PRESCRIBED_CILIA, wall)    :1887-2105
  solve_linear_system (right-preconditioned GMRES, modified Gram-Schmidt,
                       Givens rotations, warm start)  :2187-2669
and the step order of cilia_sim_main.cu:405-575 (filament::initial_guess then
mobility_solver::compute_velocities).  The mobility product comes from the C
restatement of the wall RPY kernel (oracle/rpy_oracle.c).

Saddle vector: [3N lambda | N_fil phase rates (dynamic_phase) | N_fil angle rates (dynamic_angle)].
"""
from __future__ import annotations

import math

import numpy as np

from . import rpy_apply
from .beat import Beat, filament_kinematics, wall_frame

SEG_MOB_INV = 6.0 * math.pi  # 6 pi mu a with mu = a = 1 (config.hpp MU, RSEG)


def cyclic_cubic_spline(phase: float, table) -> float:
    """Cubic Hermite interpolation of a periodic table over one beat (mobility_solver.cpp:242-282)."""
    n = len(table)
    x = 0.5 * phase / math.pi
    x -= math.floor(x)
    x *= n
    lo = int(x)
    if lo == n:
        return float(table[0])
    up = 0 if lo == n - 1 else lo + 1
    q_lo = table[lo]
    dq_lo = (table[1] - table[0]) if lo == 0 else 0.5 * (table[up] - table[lo - 1])
    q_up = table[up]
    if up == 0:
        dq_up = table[0] - table[n - 1]
    else:
        dq_up = 0.5 * (table[0 if up == n - 1 else up + 1] - table[lo])
    t = x - lo
    t2, t3 = t * t, t * t * t
    return float(q_lo * (2 * t3 - 3 * t2 + 1) + dq_lo * (t3 - 2 * t2 + t) + q_up * (3 * t2 - 2 * t3)
                 + dq_up * (t3 - t2))


def gmres_right(matvec, precond, rhs, x0, tol, max_iter):
    """Right-preconditioned GMRES in the reference's order (mobility_solver.cpp:2187-2669): the guess is
    kept when already good enough and discarded when worse than zero; modified Gram-Schmidt, Givens
    rotations, back substitution.  Returns (solution, iterations, relative residual estimate)."""
    nrm_rhs = np.linalg.norm(rhs)
    soln = np.array(x0, dtype=np.float64, copy=True)
    if nrm_rhs == 0.0:
        return np.zeros_like(soln), 0, 0.0
    r0 = rhs - matvec(soln)
    beta0 = np.linalg.norm(r0)
    if abs(beta0) <= tol * nrm_rhs:
        return soln, 0, beta0 / nrm_rhs
    if abs(beta0) > nrm_rhs:
        soln[:] = 0.0
        beta0 = nrm_rhs
        r0 = rhs.copy()
    n = rhs.size
    Q = np.zeros((n, max_iter + 1))
    H = np.zeros((max_iter + 1, max_iter + 1))
    beta = np.zeros(max_iter + 1)
    cs = np.zeros(max_iter)
    sn = np.zeros(max_iter)
    Q[:, 0] = r0 / beta0
    beta[0] = beta0
    for it in range(1, max_iter + 1):
        w = matvec(precond(Q[:, it - 1]))
        for i in range(it):
            H[i, it - 1] = w @ Q[:, i]
            w = w - H[i, it - 1] * Q[:, i]
        qn = np.linalg.norm(w)
        H[it, it - 1] = qn
        Q[:, it] = w / qn if qn != 0 else w
        for i in range(1, it):
            t = cs[i - 1] * H[i - 1, it - 1] + sn[i - 1] * H[i, it - 1]
            H[i, it - 1] = cs[i - 1] * H[i, it - 1] - sn[i - 1] * H[i - 1, it - 1]
            H[i - 1, it - 1] = t
        a, b = H[it - 1, it - 1], H[it, it - 1]
        if b == 0.0:
            cs[it - 1], sn[it - 1] = 1.0, 0.0
        elif abs(b) > abs(a):
            t = a / b
            sn[it - 1] = (1.0 if b > 0 else -1.0) / math.sqrt(1.0 + t * t)
            cs[it - 1] = t * sn[it - 1]
        else:
            t = b / a
            cs[it - 1] = (1.0 if a > 0 else -1.0) / math.sqrt(1.0 + t * t)
            sn[it - 1] = t * cs[it - 1]
        H[it - 1, it - 1] = cs[it - 1] * a + sn[it - 1] * b
        H[it, it - 1] = 0.0
        beta[it] = -sn[it - 1] * beta[it - 1]
        beta[it - 1] = cs[it - 1] * beta[it - 1]
        rel = abs(beta[it]) / nrm_rhs
        if rel <= tol or it == max_iter:
            y = np.zeros(it)
            for i in range(it - 1, -1, -1):
                y[i] = (beta[i] - H[i, i + 1:it] @ y[i + 1:it]) / H[i, i]
            return soln + precond(Q[:, :it] @ y), it, rel
    return soln, max_iter, float("nan")


class WallCilia:
    """A wall of prescribed-shape cilia with the reference's implicit step."""

    def __init__(self, *, bases, nseg, seg_sep, shape_sequence, dt, omega0=None, phase0=None, angle0=None,
                 dynamic_phase=True, dynamic_angle=True, spring_factor=0.0, phase_refs=None, angle_refs=None,
                 s_table=None, gmres_tol=1e-6, gmres_max_iter=350, precondition=True, nthreads=0):
        self.bases = np.asarray(bases, float).reshape(-1, 3)
        self.nfil = self.bases.shape[0]
        self.nseg = nseg
        self.dl = seg_sep  # RSEG = 1
        self.fil_length = self.dl * (nseg - 1)
        self.beat = Beat(shape_sequence, nseg)
        self.R = wall_frame()
        self.dt = dt
        self.omega0 = np.full(self.nfil, 2 * math.pi) if omega0 is None else np.asarray(omega0, float)
        self.phase = np.zeros(self.nfil) if phase0 is None else np.array(phase0, float)
        self.angle = np.zeros(self.nfil) if angle0 is None else np.array(angle0, float)
        self.phase_dot = self.omega0.copy()          # filament.cpp:472
        self.angle_dot = np.zeros(self.nfil)         # filament.cpp:466
        self.dyn_phase, self.dyn_angle = bool(dynamic_phase), bool(dynamic_angle)
        self.spring_factor = spring_factor
        self.phase_refs = None if phase_refs is None else np.asarray(phase_refs, float)
        self.angle_refs = None if angle_refs is None else np.asarray(angle_refs, float)
        self.s_table = None if s_table is None else np.asarray(s_table, float)
        self.tol, self.max_iter = gmres_tol, gmres_max_iter
        self.precondition = precondition
        self.nthreads = nthreads
        self.nseg_total = self.nfil * nseg
        self.lam = np.zeros(3 * self.nseg_total)     # f_segs_host force slots (GMRES warm start)
        self.x = np.zeros((self.nseg_total, 3))
        self.kp = np.zeros((self.nseg_total, 3))
        self.ka = np.zeros((self.nseg_total, 3))
        self.s_values = np.zeros((self.nfil, nseg))
        self.size = 3 * self.nseg_total + self.nfil * (int(self.dyn_phase) + int(self.dyn_angle))

    # -- filament::initial_guess ------------------------------------------
    def initial_guess(self, nt: int):
        if nt > 0:
            self.phase = self.phase + self.phase_dot * self.dt
            self.angle = self.angle + self.angle_dot * self.dt
        for m in range(self.nfil):
            psi = self.phase[m]
            s = self.beat.s_bisection(psi) if self.s_table is None else self.beat.s_from_table(psi, self.s_table)
            self.s_values[m] = s
            x, kp, ka = filament_kinematics(self.beat, s, psi, self.angle[m], self.bases[m], self.R,
                                            self.fil_length)
            sl = slice(m * self.nseg, (m + 1) * self.nseg)
            self.x[sl], self.kp[sl], self.ka[sl] = x, kp, ka

    # -- mobility_solver::assemble_rhs ------------------------------------
    def assemble_rhs(self):
        rhs = np.zeros(self.size)
        n3 = 3 * self.nseg_total
        F = self.nfil
        L3 = self.fil_length ** 3
        for m in range(F):
            if self.dyn_angle:
                q_angle = cyclic_cubic_spline(self.phase[m], self.angle_refs) * 0.5 * self.omega0[m] / math.pi
                q_angle -= self.spring_factor * self.omega0[m] * L3 * self.angle[m]   # FENE_MODEL 0
            if self.dyn_phase:
                q_phase = cyclic_cubic_spline(self.phase[m], self.phase_refs) * 0.5 * self.omega0[m] / math.pi
                rhs[n3 + m] = -q_phase
                if self.dyn_angle:
                    rhs[n3 + F + m] = -q_angle
            else:
                sl = slice(3 * m * self.nseg, 3 * (m + 1) * self.nseg)
                rhs[sl] = self.phase_dot[m] * self.kp[m * self.nseg:(m + 1) * self.nseg].ravel()
                if self.dyn_angle:
                    rhs[n3 + m] = -q_angle
        return rhs

    # -- offsets ----------------------------------------------------------
    def _offsets(self):
        n3 = 3 * self.nseg_total
        F = self.nfil
        po = n3 if self.dyn_phase else None
        ao = (n3 + F if self.dyn_phase else n3) if self.dyn_angle else None
        return n3, po, ao

    # -- apply_preconditioner_new ------------------------------------------
    def precond(self, v):
        out = np.array(v, float)
        if not self.precondition:
            return out
        n3, po, ao = self._offsets()
        F, ns = self.nfil, self.nseg
        out[:n3] *= SEG_MOB_INV
        if po is None and ao is None:
            return out
        if po is not None:
            out[po:po + F] *= -1.0
        if ao is not None:
            out[ao:ao + F] *= -1.0
        for m in range(F):
            sl = slice(3 * m * ns, 3 * (m + 1) * ns)
            kp = self.kp[m * ns:(m + 1) * ns].ravel()
            ka = self.ka[m * ns:(m + 1) * ns].ravel()
            r1 = out[sl]
            if po is not None and ao is not None:
                c11, c22, c12 = kp @ kp, ka @ ka, ka @ kp
                p = out[po + m] - kp @ r1
                a = out[ao + m] - ka @ r1
                det = c11 * c22 - c12 * c12
                out[po + m] = (p * c22 / det + a * (-c12 / det)) / SEG_MOB_INV
                out[ao + m] = (p * (-c12 / det) + a * c11 / det) / SEG_MOB_INV
                out[sl] = r1 + SEG_MOB_INV * (out[po + m] * kp + out[ao + m] * ka)
            elif po is not None:
                out[po + m] = (out[po + m] - kp @ r1) / ((kp @ kp) * SEG_MOB_INV)
                out[sl] = r1 + SEG_MOB_INV * out[po + m] * kp
            else:
                out[ao + m] = (out[ao + m] - ka @ r1) / ((ka @ ka) * SEG_MOB_INV)
                out[sl] = r1 + SEG_MOB_INV * out[ao + m] * ka
        return out

    # -- line-patch block-Jacobi preconditioner --------------------------------
    # Not a reference routine: the engine's CF_PRECOND_LINE restated in FP64 for
    # its parity tests.  Patches come from line_patches(); each patch's saddle
    # block (the system_matrix_mult_new operator restricted to the patch) is
    # inverted exactly.
    def patch_block(self, fils):
        """Dense saddle block of the filaments `fils`, per-filament order [3*nseg lambda | rates]."""
        ns = self.nseg
        n3, po, ao = self._offsets()
        nr = int(po is not None) + int(ao is not None)
        nbf = 3 * ns + nr
        segs = np.concatenate([np.arange(f * ns, (f + 1) * ns) for f in fils])
        x = self.x[segs]
        nl = len(segs)
        M = np.zeros((3 * nl, 3 * nl))
        for c in range(3 * nl):
            f = np.zeros((nl, 3))
            f.flat[c] = 1.0
            M[:, c] = rpy_apply(x, x, f, wall=1, vdof=3, fdof=3, self_by_index=True, nthreads=self.nthreads).ravel()
        nf = len(fils)
        A = np.zeros((nbf * nf, nbf * nf))
        for a in range(nf):
            for b in range(nf):
                A[nbf * a:nbf * a + 3 * ns, nbf * b:nbf * b + 3 * ns] = M[3 * ns * a:3 * ns * (a + 1),
                                                                         3 * ns * b:3 * ns * (b + 1)]
            cols = []
            if po is not None:
                cols.append(self.kp[fils[a] * ns:(fils[a] + 1) * ns].ravel())
            if ao is not None:
                cols.append(self.ka[fils[a] * ns:(fils[a] + 1) * ns].ravel())
            for q, k in enumerate(cols):
                A[nbf * a:nbf * a + 3 * ns, nbf * a + 3 * ns + q] = -k
                A[nbf * a + 3 * ns + q, nbf * a:nbf * a + 3 * ns] = -k
        return A

    def patch_rows(self, fils):
        """Saddle-vector rows of the patch unknowns, in the order of patch_block."""
        ns = self.nseg
        n3, po, ao = self._offsets()
        rows = []
        for f in fils:
            rows.extend(range(3 * ns * f, 3 * ns * (f + 1)))
            if po is not None:
                rows.append(po + f)
            if ao is not None:
                rows.append(ao + f)
        return np.asarray(rows)

    def line_patch_precond(self, v, line_patch=32):
        out = np.zeros(self.size)
        v = np.asarray(v, float)
        for fils in line_patches(self.bases, line_patch):
            rows = self.patch_rows(fils)
            out[rows] = np.linalg.solve(self.patch_block(fils), v[rows])
        return out

    def learned_features(self, v):
        """Features of the learned preconditioner's network for vector v (not a reference routine):
        [own force rows | 2 rate rows | neighbour-mean force rows] / s, then the shape relative to the
        base over the filament length; returns (X [F, 9*nseg+2], s [F])."""
        ns, F = self.nseg, self.nfil
        n3, po, ao = self._offsets()
        v = np.asarray(v, float)
        lam = v[:n3].reshape(F, 3 * ns)
        rates = np.zeros((F, 2))
        if po is not None:
            rates[:, 0] = v[po:po + F]
        if ao is not None:
            rates[:, 1] = v[ao:ao + F]
        nbr = line_neighbours(self.bases)
        mean = np.zeros_like(lam)
        for m in range(F):
            ids = [k for k in nbr[m] if k >= 0]
            if ids:
                mean[m] = lam[ids].mean(0)
        s = np.sqrt((lam ** 2).sum(1) + (rates ** 2).sum(1) + (mean ** 2).sum(1))
        si = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
        shape = (self.x.reshape(F, ns, 3) - self.bases[:, None, :]).reshape(F, 3 * ns) / self.fil_length
        X = np.concatenate([lam * si[:, None], rates * si[:, None], mean * si[:, None], shape], 1)
        return X, s

    # -- mobility product (Mss_mult, wall, 3x3) -----------------------------
    def mobility(self, lam):
        f = np.asarray(lam, float).reshape(-1, 3)
        return rpy_apply(self.x, self.x, f, wall=1, vdof=3, fdof=3, self_by_index=True,
                         nthreads=self.nthreads).ravel()

    # -- system_matrix_mult_new ----------------------------------------------
    def matvec(self, v):
        v = np.asarray(v, float)
        n3, po, ao = self._offsets()
        F, ns = self.nfil, self.nseg
        out = np.zeros(self.size)
        lam = v[:n3]
        out[:n3] = self.mobility(lam)
        for m in range(F):
            sl = slice(3 * m * ns, 3 * (m + 1) * ns)
            kp = self.kp[m * ns:(m + 1) * ns].ravel()
            ka = self.ka[m * ns:(m + 1) * ns].ravel()
            if po is not None:
                out[sl] -= v[po + m] * kp
                out[po + m] = -(kp @ lam[sl])
            if ao is not None:
                out[sl] -= v[ao + m] * ka
                out[ao + m] = -(ka @ lam[sl])
        return out

    # -- solution vector <-> state ----------------------------------------
    def _pack_solution(self):
        n3, po, ao = self._offsets()
        s = np.zeros(self.size)
        s[:n3] = self.lam
        if po is not None:
            s[po:po + self.nfil] = self.phase_dot
        if ao is not None:
            s[ao:ao + self.nfil] = self.angle_dot
        return s

    def _unpack_solution(self, s):
        n3, po, ao = self._offsets()
        self.lam = s[:n3].copy()
        if po is not None:
            self.phase_dot = s[po:po + self.nfil].copy()
        if ao is not None:
            self.angle_dot = s[ao:ao + self.nfil].copy()

    # -- solve_linear_system ------------------------------------------------
    def solve(self, rhs):
        """Right-preconditioned GMRES exactly as the reference orders it; returns (iters, relres)."""
        if np.linalg.norm(rhs) == 0.0:
            self.lam[:] = 0.0
            if self.dyn_phase:
                self.phase_dot[:] = 0.0
            if self.dyn_angle:
                self.angle_dot[:] = 0.0
            return 0, 0.0
        soln, it, rel = gmres_right(self.matvec, self.precond, rhs, self._pack_solution(), self.tol,
                                    min(self.size, self.max_iter))
        self._unpack_solution(soln)
        return it, rel

    # -- one implicit step (cilia_sim_main.cu:405-416) -------------------------
    def step(self, nt: int):
        self.initial_guess(nt)
        rhs = self.assemble_rhs()
        return self.solve(rhs)

    def generalised_forces(self):
        """K_phase^T lambda and K_angle^T lambda per filament (cilia_sim_main.cu:420-440)."""
        lam = self.lam.reshape(-1, 3)
        qp = np.array([np.sum(self.kp[m * self.nseg:(m + 1) * self.nseg] * lam[m * self.nseg:(m + 1) * self.nseg])
                       for m in range(self.nfil)])
        qa = np.array([np.sum(self.ka[m * self.nseg:(m + 1) * self.nseg] * lam[m * self.nseg:(m + 1) * self.nseg])
                       for m in range(self.nfil)])
        return qp, qa

    def tips(self):
        return self.x.reshape(self.nfil, self.nseg, 3)[:, -1, :].copy()


def line_neighbours(bases):
    """[F, 2] previous / next filament along each lattice line (equal base x, sorted by y), -1 at the ends."""
    b = np.asarray(bases, float).reshape(-1, 3)
    order = sorted(range(b.shape[0]), key=lambda i: (b[i, 0], b[i, 1]))
    nbr = -np.ones((b.shape[0], 2), int)
    for q, i in enumerate(order):
        x0 = b[i, 0]
        if q > 0 and abs(b[order[q - 1], 0] - x0) <= 1e-6 * (1.0 + abs(x0)):
            nbr[i, 0] = order[q - 1]
        if q + 1 < len(order) and abs(b[order[q + 1], 0] - x0) <= 1e-6 * (1.0 + abs(x0)):
            nbr[i, 1] = order[q + 1]
    return nbr


def line_patches(bases, line_patch=32):
    """Filament groups of the line-patch preconditioner: filaments with equal base x (a
    lattice line along y, the beat direction of the wall frame) sorted by y, cut into runs
    of at most `line_patch` filaments of near-equal length (the longer runs first)."""
    b = np.asarray(bases, float).reshape(-1, 3)
    order = sorted(range(b.shape[0]), key=lambda i: (b[i, 0], b[i, 1]))
    out, s0 = [], 0
    while s0 < len(order):
        x0 = b[order[s0], 0]
        s1 = s0 + 1
        while s1 < len(order) and abs(b[order[s1], 0] - x0) <= 1e-6 * (1.0 + abs(x0)):
            s1 += 1
        L = s1 - s0
        c = -(-L // line_patch)
        base, extra = divmod(L, c)
        pos = s0
        for q in range(c):
            sz = base + (1 if q < extra else 0)
            out.append(order[pos:pos + sz])
            pos += sz
        s0 = s1
    return out


def write_generalised_forces_run(shape_sequence: int, nseg: int = 20, seg_sep: float = 2.6, steps: int = 300,
                                 tol: float = 1e-4, s_table=None):
    """The reference's WRITE_GENERALISED_FORCES run: one filament, prescribed phase speed 2 pi,
    no dynamic phase/angle, base at 0.5*DL (cilia_sim_main.cu:101-140, 318-338, 420-440).
    Returns (phase forces [steps], angle forces [steps], s-values [steps, nseg])."""
    dl = seg_sep
    sim = WallCilia(bases=[[0.0, 0.0, 0.5 * dl]], nseg=nseg, seg_sep=seg_sep, shape_sequence=shape_sequence,
                    dt=1.0 / steps, dynamic_phase=False, dynamic_angle=False, gmres_tol=tol, s_table=s_table)
    qp, qa, sv = np.zeros(steps), np.zeros(steps), np.zeros((steps, nseg))
    for nt in range(steps):
        sim.step(nt)
        q1, q2 = sim.generalised_forces()
        qp[nt], qa[nt] = q1[0], q2[0]
        sv[nt] = sim.s_values[0]
    return qp, qa, sv
