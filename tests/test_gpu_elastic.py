"""GPU tests of the elastic-filament step (cf_elastic) through the C ABI.

Oracle: the reference's own host step code for instability-driven cilia on a wall
(tests/golden/ref_elastic_2x2_80a.npz, and ref_elastic_2x2_2p1a.npz with touching cilia, where the
segment-segment barrier forces act; make_elastic_golden.py).  The approximate
Jacobian is FP64 throughout and is compared at 1e-10; the residual of the first
evaluation carries the FP32 pair mobility (1e-5 of its largest entry).  The trajectory:
the follower force buckles the filaments, an instability that amplifies any difference,
so the positions are compared over the run with a tolerance that grows with it: FP32
pair sums and Broyden's stopping test (TOL 1e-4) perturb each step by ~1e-6 L.
"""
from pathlib import Path

import numpy as np
import pytest

from cufcm_fil_b200 import _lib, workloads
from cufcm_fil_b200.elastic import ElasticCiliaSimulation

pytestmark = pytest.mark.gpu

EL = np.load(Path(__file__).resolve().parent / "golden" / "ref_elastic_2x2_80a.npz")
ELC = np.load(Path(__file__).resolve().parent / "golden" / "ref_elastic_2x2_2p1a.npz")
ELP = np.load(Path(__file__).resolve().parent / "golden" / "ref_elastic_jinv_probes.npz")
L = 2.6 * 20  # FIL_LENGTH = DL NSEG for elastic filaments


def make(nx, spacing, **kw):
    bases = workloads.lattice_bases(nx * nx, nx, spacing, 1.3)
    return ElasticCiliaSimulation(bases=bases, nseg=20, seg_sep=2.6, dt=float(EL["period"]) / 300, **kw)


def test_first_evaluation_and_jacobian_match_reference():
    with make(1, 80.0) as sim:
        err = sim.first_evaluation(0)
        jinv = sim.jacobian_inverse(0)
    ref = EL["jinv0"]
    assert np.linalg.norm(jinv - ref) / np.linalg.norm(ref) < 1e-10
    np.testing.assert_allclose(err, EL["err0"], rtol=0, atol=1e-5 * np.abs(EL["err0"]).max())


@pytest.mark.parametrize("nseg", [14, 20, 24])
def test_jacobian_inverse_every_block_size(nseg):
    """The device inversion has one form per block size class (84, 120, 144 unknowns here): each matches
    the reference's invert_approx_jacobian through seeded probes."""
    bases = workloads.lattice_bases(1, 1, 80.0, 1.3)
    with ElasticCiliaSimulation(bases=bases, nseg=nseg, seg_sep=2.6, dt=float(ELP["period"]) / 300) as sim:
        sim.first_evaluation(0)
        jinv = sim.jacobian_inverse(0)
    v = np.random.default_rng(5).standard_normal((6 * nseg, 4))
    ref = ELP[f"p{nseg}"]
    assert np.linalg.norm(jinv @ v - ref) / np.linalg.norm(ref) < 1e-10
    assert abs(np.linalg.norm(jinv) / float(ELP[f"norm{nseg}"]) - 1.0) < 1e-10


def test_trajectory_follows_reference():
    saved = list(EL["saved_steps"])
    worst = []
    iters = []
    with make(int(EL["nx"]), float(EL["spacing"])) as sim:
        for nt in range(int(EL["steps"])):
            iters.append(sim.step(nt))
            if nt in saved:
                x = sim.segments()[0]
                worst.append(np.abs(x - EL["x"][saved.index(nt)]).max() / L)
        st = sim.stats()
    worst = np.array(worst)
    it_ref = EL["iterations"]
    diff = np.array(iters) - it_ref
    print(f"elastic 2x2, 300 steps: position error / L at steps 0, 100, 200, 290: "
          f"{worst[0]:.2e} {worst[10]:.2e} {worst[20]:.2e} {worst[-1]:.2e}; Broyden iterations "
          f"{np.mean(iters):.2f} (reference {it_ref.mean():.2f}), max {st['max']}; per-step difference "
          f"{diff.min()}..{diff.max()}, equal on {np.mean(diff == 0):.0%} of the steps")
    assert st["steps"] == 300 and st["total"] == sum(iters)
    # The stopping test (TOL 1e-4 on every residual entry) sees the FP32 pair sums: a step may stop an
    # iteration or a few earlier or later than the reference's, the counts agree on average.
    assert iters[0] == it_ref[0] and abs(np.mean(iters) - it_ref.mean()) < 0.1 * it_ref.mean()
    assert worst[:11].max() < 1e-4   # through step 100, before the buckling grows
    assert worst.max() < 1e-2


def test_bad_configuration_is_rejected():
    with pytest.raises(_lib.CufilError):
        ElasticCiliaSimulation(bases=[[0.0, 0.0, 1.3]], nseg=10)          # the perturbations need 13 segments
    with pytest.raises(_lib.CufilError):
        ElasticCiliaSimulation(bases=[[0.0, 0.0, 1.3]], nseg=20, ic_type=2)  # type 2 needs the perturbations


def test_broyden_cap_and_non_finite_state_are_reported():
    # one Broyden iteration cannot reach TOL from the straight start: CF_NOT_CONVERGED, as the reference stops
    with make(1, 80.0, max_broyden_iter=1) as sim:
        with pytest.raises(_lib.CufilError) as e:
            sim.step(0)
        assert e.value.code == _lib.CF_NOT_CONVERGED
    # a NaN perturbation makes the first residual non-finite: CF_NONFINITE, and the handle stays usable
    pert = np.zeros((1, 2, 3))
    pert[0, 0, 0] = np.nan
    with make(1, 80.0, ic_type=2, perturbations=pert) as sim:
        with pytest.raises(_lib.CufilError) as e:
            sim.step(0)
        assert e.value.code == _lib.CF_NONFINITE
        sim.stats()


def test_touching_cilia_follow_reference():
    # 2 x 2 lattice at 2.1a: the bases of neighbouring cilia are inside the barrier range 2.2a, so the
    # segment-segment barrier forces act from the first evaluation (20 steps of the reference's own step).
    # The barrier is stiff: Broyden's method takes 40 iterations at step 0 in the reference.
    iters, worst = [], []
    with make(int(ELC["nx"]), float(ELC["spacing"])) as sim:
        for nt in range(int(ELC["steps"])):
            iters.append(sim.step(nt))
            x = sim.segments()[0]
            worst.append(np.abs(x - ELC["x"][nt]).max() / L)
    it_ref = ELC["iterations"]
    print(f"touching cilia, 20 steps: position error / L at steps 0, 9, 19: {worst[0]:.2e} {worst[9]:.2e} "
          f"{worst[19]:.2e}; Broyden iterations {iters} (reference {it_ref.tolist()})")
    assert max(worst) < 1e-5
    assert abs(iters[0] - it_ref[0]) <= 2 and abs(np.mean(iters) - it_ref.mean()) < 0.15 * it_ref.mean()
