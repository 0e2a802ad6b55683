"""The FP64 restatement of the reference's flow-field kernel (oracle/flow.py): physical checks, no GPU."""
import numpy as np

from oracle import flow


def _sources(n, seed, torques=True):
    rng = np.random.default_rng(seed)
    xs = rng.uniform([-20, -20, 1.5], [20, 20, 30], (n, 3))
    fs = np.zeros((n, 6))
    fs[:, :3] = rng.standard_normal((n, 3))
    if torques:
        fs[:, 3:] = rng.standard_normal((n, 3))
    return xs, fs


def test_blake_image_gives_no_slip_on_the_wall():
    # Without blobs the segment Stokeslets carry Blake's image system: zero velocity on z = 0
    # (segment torques have no image in the reference, so they are zero here).
    xs, fs = _sources(40, 1, torques=False)
    xf = np.random.default_rng(2).uniform([-50, -50, 0], [50, 50, 0], (30, 3))
    v = flow.flow_velocities(xf, xs, fs, n_seg_per_body=40)
    ref = np.abs(flow.flow_velocities(xf + [0, 0, 5.0], xs, fs, n_seg_per_body=40)).max()
    assert np.abs(v).max() < 1e-12 * ref


def test_free_space_stokeslet_and_linearity():
    # One blob (no image): u = (1/(8 pi mu)) (f/r + r (r.f)/r^3)
    xb = np.array([[1.0, 2.0, 3.0]])
    fb = np.array([[0.3, -0.2, 0.5]])
    xf = np.array([[4.0, -1.0, 7.0]])
    r = xf[0] - xb[0]
    d = np.linalg.norm(r)
    u = (fb[0] / d + r * (r @ fb[0]) / d ** 3) / (8 * np.pi * 2.0)
    v = flow.flow_velocities(xf, np.zeros((0, 3)), np.zeros((0, 6)), xb, fb, n_seg_per_body=1, n_blob_per_body=1,
                             mu=2.0)
    np.testing.assert_allclose(v[0], u, rtol=1e-14)
    xs, fs = _sources(25, 3)
    xf = np.random.default_rng(4).uniform(-30, 30, (10, 3)) + [0, 0, 40]
    a = flow.flow_velocities(xf, xs, fs, n_seg_per_body=25)
    b = flow.flow_velocities(xf, xs, 2.5 * fs, n_seg_per_body=25)
    np.testing.assert_allclose(b, 2.5 * a, rtol=1e-12)


def test_removing_the_net_force_makes_the_far_field_decay_faster():
    # With remove_net_force each source's Stokeslet is replaced by its difference from a Stokeslet
    # at the body centre: far from a compact body the velocity decays faster than 1/r.
    rng = np.random.default_rng(5)
    xb = rng.uniform(-3, 3, (50, 3))
    fb = rng.standard_normal((50, 3))
    body = np.zeros((1, 3))
    far = [np.array([[0.0, 0.0, R]]) for R in (200.0, 400.0)]
    v = [np.linalg.norm(flow.flow_velocities(x, np.zeros((0, 3)), np.zeros((0, 6)), xb, fb, body, n_seg_per_body=1,
                                             n_blob_per_body=50, remove_net_force=True)) for x in far]
    assert v[1] / v[0] < 0.3   # ~1/r^2 (4x drop), not ~1/r (2x)
