"""The free swimmer's oracle (oracle/swim.py) against the reference's own step code.

tests/golden/ref_swim_12fil_642blob.npz is a 300-step run of the reference's host step
code for 12 prescribed cilia on a free sphere of 642 blobs (make_swim_golden.py).  The
oracle restates the body branches of system_matrix_mult_new / apply_preconditioner_new,
make_precon_mat, the filament frames and the body update; it must follow that trajectory
to rounding.  The preconditioner is also checked for what it is built to be: the exact
inverse of the saddle matrix when the mobility is its diagonal 1/(6 pi) part.
"""
from pathlib import Path

import numpy as np

from oracle import swim
from cufcm_fil_b200.swim import sphere_geometry

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")
SWIM = np.load(Path(__file__).resolve().parent / "golden" / "ref_swim_12fil_642blob.npz")


def make_oracle():
    geo = sphere_geometry(SWIM["fil_normals"], SWIM["blob_normals"], ar=float(SWIM["ar"]))
    return swim.Swimmer(fil_refs=geo.fil_refs, fil_dirs=geo.fil_dirs, blob_refs=geo.blob_refs, nseg=20, seg_sep=2.6,
                        dt=1 / 300, phase0=SWIM["phase0"], angle0=SWIM["angle0"], phase_refs=GOLD["fb_phase"],
                        angle_refs=GOLD["fb_angle"], s_table=SWIM["s_table"])


def test_oracle_follows_the_reference_swimmer():
    s = make_oracle()
    L = 2.6 * 19
    for nt in range(20):
        np.testing.assert_allclose(s.body_x, SWIM["body_x"][nt], rtol=0, atol=1e-11)
        it, rel = s.step(nt)
        assert it == SWIM["iterations"][nt] and rel <= 1e-6
        assert np.abs(s.tips() - SWIM["tips"][nt]).max() / L < 1e-12
        np.testing.assert_allclose(s.body_v, SWIM["body_v"][nt], rtol=1e-10, atol=1e-11)
        np.testing.assert_allclose(s.phase_dot, SWIM["phase_dot"][nt], rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(s.angle_dot, SWIM["angle_dot"][nt], rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(s.body_q, SWIM["body_q"][nt + 1], rtol=0, atol=1e-14)


def test_preconditioner_inverts_the_diagonal_mobility_system():
    rng = np.random.default_rng(3)
    nseg, F, B = 5, 3, 7
    xs = rng.normal(0, 10, (F * nseg, 3))
    xb = rng.normal(0, 10, (B, 3))
    bx = rng.normal(0, 1, 3)
    kp, ka = rng.normal(size=(F * nseg, 3)), rng.normal(size=(F * nseg, 3))
    n = 3 * (F * nseg + B) + 6 + 2 * F

    def a_diag(v):  # the saddle product with M replaced by I / (6 pi)
        out = swim.matvec(xs, xb, bx, kp, ka, np.zeros(n), nseg)  # geometry-only rows, mobility part below
        fs, fb, V, W, ph, an = swim._split(v, F * nseg, B, F)
        ds, db = xs - bx, xb - bx
        rate = np.repeat(ph, nseg)[:, None] * kp + np.repeat(an, nseg)[:, None] * ka
        out[:3 * F * nseg] = (fs / swim.MOB - V - np.cross(W, ds) - rate).ravel()
        out[3 * F * nseg:3 * (F * nseg + B)] = (fb / swim.MOB - V - np.cross(W, db)).ravel()
        o = 3 * (F * nseg + B)
        out[o:o + 3] = -(fs.sum(0) + fb.sum(0))
        out[o + 3:o + 6] = -(np.cross(ds, fs).sum(0) + np.cross(db, fb).sum(0))
        out[o + 6:o + 6 + F] = -(kp * fs).reshape(F, -1).sum(1)
        out[o + 6 + F:] = -(ka * fs).reshape(F, -1).sum(1)
        return out

    A = np.stack([a_diag(e) for e in np.eye(n)], axis=1)
    P = np.stack([swim.precond(xs, xb, bx, kp, ka, e, nseg) for e in np.eye(n)], axis=1)
    np.testing.assert_allclose(A @ P, np.eye(n), atol=1e-9)


def test_filament_frame_on_the_wall_is_the_wall_frame():
    from oracle.beat import quat_rot, wall_frame
    np.testing.assert_allclose(quat_rot(*swim.filament_frame([0.0, 0.0, 1.0])), wall_frame(), atol=1e-15)
