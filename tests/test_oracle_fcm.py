"""CPU checks of the FCM oracle (restatement of the reference's cuFCM, oracle/fcm.py).

The fast FCM mobility is symmetric, and for well-separated particles in a
large periodic box it approaches the unbounded RPY mobility (the difference is
the periodic images and the Gaussian-vs-RPY near field, a few percent here).
"""
import numpy as np

import oracle
from oracle import fcm


def _particles(n, box, seed, min_dist=4.0):
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n:
        p = rng.uniform(0.3 * box, 0.7 * box, 3)
        if all(np.linalg.norm(p - q) > min_dist for q in pts):
            pts.append(p)
    return np.array(pts)


def test_fcm_mobility_is_symmetric():
    p = fcm.FcmParams(nx=32, ny=32, nz=32, boxsize=64.0, alpha=1.0, beta=8.0, eta=5.0)
    Y = _particles(12, 64.0, 1)
    rng = np.random.default_rng(2)
    F, G = rng.standard_normal((12, 3)), rng.standard_normal((12, 3))
    a = np.sum(G * fcm.fcm_apply(Y, F, p))
    b = np.sum(F * fcm.fcm_apply(Y, G, p))
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))


def test_fcm_approaches_unbounded_rpy_in_a_large_box():
    p = fcm.FcmParams(nx=64, ny=64, nz=64, boxsize=256.0, alpha=1.0, beta=10.0, eta=6.0)
    Y = _particles(16, 256.0, 3, min_dist=6.0)
    F = np.random.default_rng(4).standard_normal((16, 3))
    v_fcm = fcm.fcm_apply(Y, F, p)
    v_rpy = oracle.rpy_apply(Y, Y, F, wall=0, vdof=3, fdof=3)
    assert oracle.rel_l2(v_fcm, v_rpy) < 0.05


def test_single_particle_self_mobility_is_stokes_up_to_images():
    # the periodic correction of a single sphere is -2.837 a/L (Hasimoto); L = 256 a
    p = fcm.FcmParams(nx=64, ny=64, nz=64, boxsize=256.0)
    v = fcm.fcm_apply(np.array([[100.0, 120.0, 130.0]]), np.array([[1.0, 0.0, 0.0]]), p)
    stokes = 1.0 / (6 * np.pi)
    assert abs(v[0, 0] / stokes - (1 - 2.837 / 256.0)) < 5e-3
    assert abs(v[0, 1]) < 1e-6 * stokes and abs(v[0, 2]) < 1e-6 * stokes
