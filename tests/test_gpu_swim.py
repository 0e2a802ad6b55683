"""GPU tests of the free swimmer (cf_swim) through the C ABI.

Operators: for the geometry the engine built at step 0, the saddle product and the
preconditioner on random vectors against the FP64 oracle (oracle/swim.py) evaluated on
the engine's own FP64 positions and velocity directions: the preconditioner is FP64
throughout (1e-10), the product carries the FP32 pair sums of the tile kernel (relative
L2 below 1e-5, the mobility contract).  Trajectory: 300 steps (one beat period) of 12
cilia on a free sphere of 642 blobs against the reference's own step code
(tests/golden/ref_swim_12fil_642blob.npz).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import swim as oswim
from cufcm_fil_b200 import _lib
from cufcm_fil_b200.swim import CiliatedSwimmer, sphere_geometry

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")
SWIM = np.load(Path(__file__).resolve().parent / "golden" / "ref_swim_12fil_642blob.npz")
L = 2.6 * 19


def make_swimmer(**kw):
    geo = sphere_geometry(SWIM["fil_normals"], SWIM["blob_normals"], ar=float(SWIM["ar"]))
    return CiliatedSwimmer(geometry=geo, nseg=20, seg_sep=2.6, dt=1 / 300, phase0=SWIM["phase0"],
                           angle0=SWIM["angle0"], phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"],
                           s_table=SWIM["s_table"], gmres_tol=1e-6, **kw)


def test_operators_match_oracle():
    with make_swimmer() as s:
        bx = s.state()["body_x"]
        s.step(0)
        xs, xb, _, _ = s.particles()
        kp, ka = s.directions()
        rng = np.random.default_rng(5)
        for _ in range(3):
            v = rng.standard_normal(s.size)
            a = s.system_matrix_mult_new(v)
            a_ref = oswim.matvec(xs, xb, bx, kp, ka, v, 20)
            assert np.linalg.norm(a - a_ref) / np.linalg.norm(a_ref) < 1e-5
            p = s.apply_preconditioner_new(v)
            p_ref = oswim.precond(xs, xb, bx, kp, ka, v, 20)
            np.testing.assert_allclose(p, p_ref, rtol=1e-10, atol=1e-10 * np.abs(p_ref).max())


def test_first_step_geometry_matches_reference():
    with make_swimmer() as s:
        s.step(0)
        assert np.abs(s.tips() - SWIM["tips"][0]).max() / L < 1e-12


def test_300_steps_follow_the_reference_swimmer():
    # One beat period; the body swims ~5.6a along z.  The FP32 pair sums perturb each solve at
    # the 1e-7 level; the tolerance below bounds their effect over the period.
    TOL = 2e-4
    worst = dict(tip=0.0, body_x=0.0, body_v=0.0, phase=0.0)
    with make_swimmer() as s:
        for nt in range(int(SWIM["steps"])):
            st = s.state()
            worst["body_x"] = max(worst["body_x"], np.abs(st["body_x"] - SWIM["body_x"][nt]).max() / L)
            res = s.step(nt)
            assert res.status == _lib.CF_OK and res.relative_residual <= 1e-6
            assert abs(res.iterations - int(SWIM["iterations"][nt])) <= 1
            st = s.state()
            worst["tip"] = max(worst["tip"], np.abs(s.tips() - SWIM["tips"][nt]).max() / L)
            vref = SWIM["body_v"][nt]
            worst["body_v"] = max(worst["body_v"], np.abs(st["body_v"] - vref).max() / np.abs(vref).max())
            worst["phase"] = max(worst["phase"], np.abs(st["phase"] - SWIM["phase"][nt]).max())
    print("free swimmer, 300 steps: worst " + ", ".join(f"{k} {v:.2e}" for k, v in worst.items()))
    assert worst["tip"] < TOL and worst["body_x"] < TOL and worst["phase"] < 2 * np.pi * TOL
    assert worst["body_v"] < 1e-3


def test_bad_configuration_is_rejected():
    geo = sphere_geometry(SWIM["fil_normals"][:2], SWIM["blob_normals"][:4], ar=3.0)
    with pytest.raises(_lib.CufilError):
        CiliatedSwimmer(geometry=geo, nseg=1, phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"])
    with pytest.raises(_lib.CufilError):
        CiliatedSwimmer(geometry=geo, nseg=20)  # no generalised-force tables


def test_non_finite_state_is_reported():
    phase0 = np.array(SWIM["phase0"], float)
    phase0[3] = np.nan
    geo = sphere_geometry(SWIM["fil_normals"], SWIM["blob_normals"], ar=float(SWIM["ar"]))
    with CiliatedSwimmer(geometry=geo, phase0=phase0, angle0=SWIM["angle0"], phase_refs=GOLD["fb_phase"],
                         angle_refs=GOLD["fb_angle"], s_table=SWIM["s_table"]) as s:
        with pytest.raises(_lib.CufilError) as e:
            s.step(0)
        assert e.value.code == _lib.CF_NONFINITE
