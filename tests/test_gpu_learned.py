"""GPU tests of the learned preconditioner (CF_PRECOND_LEARNED) through the C ABI.

Features are checked against the oracle's restatement (float32 storage: 1e-6
relative); training uses the library's own kernels; the comparison with the
block-diagonal preconditioner on a state the network has not seen is measured
(gain = block-diagonal iterations / learned iterations) and compare's choice is
checked against it.  A gain below 1 is an expected failure that carries the
measured number: the filament-local correction has so far not beaten the
preconditioner it corrects.  Whatever the network does, a converged learned
step satisfies the oracle's FP64 system (the residual is formed with the exact
operator).
"""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import implicit
from cufcm_fil_b200 import _lib, learned, workloads
from cufcm_fil_b200.mlp import FilamentMLP
from cufcm_fil_b200.sim import WallCiliaSimulation

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")
NX = 6


def _args(seed):
    F = NX * NX
    rng = np.random.default_rng(seed)
    return dict(bases=workloads.lattice_bases(F, NX, 20.0, 1.3), nseg=20, seg_sep=2.6, dt=1 / 300,
                phase0=rng.uniform(0, 2 * np.pi, F), angle0=rng.normal(0, 0.05, F), spring_factor=0.01,
                phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"], gmres_tol=1e-6)


def make_sim(seed, precond):
    return WallCiliaSimulation(precond=precond, **_args(seed))


def test_features_match_oracle():
    with make_sim(3, _lib.CF_PRECOND_BLOCK_DIAG) as sim:
        sim.initial_guess(0)
        cpu = implicit.WallCilia(shape_sequence=1, **_args(3))
        cpu.initial_guess(0)
        v = np.random.default_rng(1).standard_normal(sim.size)
        X = sim.features(v)
        Xr, _ = cpu.learned_features(v)
        assert X.shape == Xr.shape == (NX * NX, 9 * 20 + 2)
        np.testing.assert_allclose(X, Xr, rtol=2e-6, atol=2e-6)


def test_collected_pairs_shape_and_values():
    with make_sim(4, _lib.CF_PRECOND_BLOCK_DIAG) as sim:
        x, t = sim.collect_pairs(0, 30)
        r = sim.last_solve()
    F = NX * NX
    assert x.shape[0] == t.shape[0] == 30 * F and r.iterations >= 30
    assert x.shape[1] == 182 and t.shape[1] == 62
    assert bool(x.isfinite().all()) and bool(t.isfinite().all())


def test_trained_network_gain_is_measured_and_decided():
    x, t = learned.collect(make_sim, seeds=(10, 11, 12), max_pairs=120)
    with FilamentMLP(182, 256, 62, max_batch=4096, seed=0) as net:
        losses = learned.train(net, x, t, steps=1500, batch=2048, lr=1e-3, report_every=500)
        assert losses[-1] < losses[0]
        cmp = learned.compare(make_sim, 99, net)
        print(f"held-out state: block-diagonal {cmp.block_diagonal_iterations} iterations, learned "
              f"{cmp.learned_iterations} at weight {cmp.weight} (status {cmp.learned_status}), gain "
              f"{cmp.gain:.2f}; by weight {cmp.by_weight}; losses {losses}")
        assert cmp.block_diagonal_status in (_lib.CF_OK, _lib.CF_NOT_CONVERGED)
        assert cmp.use_learned == (cmp.learned_status == _lib.CF_OK and cmp.gain > 1.0)
        # a converged learned step satisfies the FP64 system of the oracle
        with make_sim(99, _lib.CF_PRECOND_LEARNED) as sim:
            sim.set_network(net)
            sim.set_network_weight(cmp.weight)
            res = sim.step(0)
            if res.status == _lib.CF_OK:
                cpu = implicit.WallCilia(shape_sequence=1, **_args(99))
                cpu.initial_guess(0)
                st = sim.state()
                _, fs = sim.segments()
                sol = np.concatenate([fs.reshape(-1, 6)[:, :3].astype(np.float64).ravel(), st["phase_dot"],
                                      st["angle_dot"]])
                rhs = cpu.assemble_rhs()
                assert np.linalg.norm(rhs - cpu.matvec(sol)) / np.linalg.norm(rhs) < 2e-5
        if cmp.gain < 1.0:
            pytest.xfail(f"the learned correction loses on the held-out state: gain {cmp.gain:.2f} "
                         f"({cmp.block_diagonal_iterations} -> {cmp.learned_iterations} iterations)")
        assert cmp.gain >= 1.0


def test_learned_handle_needs_a_network():
    with make_sim(5, _lib.CF_PRECOND_LEARNED) as sim:
        with pytest.raises(_lib.CufilError):
            sim.step(0)
        with FilamentMLP(40, 16, 8, max_batch=64) as wrong:
            with pytest.raises(_lib.CufilError):
                sim.set_network(wrong)


def test_zero_weight_learned_line_equals_line_patches():
    # With the correction weight 0 the learned-line mode is the line-patch preconditioner run in
    # flexible GMRES: the same Krylov space, so the same iteration count (to one rounding step).
    with make_sim(7, _lib.CF_PRECOND_LINE) as sim:
        r_line = sim.step(0)
    with FilamentMLP(182, 64, 62, max_batch=256, seed=1) as net, make_sim(7, _lib.CF_PRECOND_LEARNED_LINE) as sim:
        sim.set_network(net)
        sim.set_network_weight(0.0)
        r = sim.step(0)
    assert r.status == r_line.status == _lib.CF_OK
    assert abs(r.iterations - r_line.iterations) <= 1


def test_network_on_top_of_line_patches_is_measured():
    # Pairs from line-patch runs (the correction learns what the patches miss: the coupling between
    # lattice lines); held-out state; the gain is line-patch iterations / learned-line iterations.
    x, t = learned.collect(make_sim, seeds=(20, 21, 22), max_pairs=60, base=_lib.CF_PRECOND_LINE)
    assert x.shape[0] > 0 and bool(t.isfinite().all())
    with FilamentMLP(182, 256, 62, max_batch=4096, seed=0) as net:
        losses = learned.train(net, x, t, steps=1500, batch=2048, lr=1e-3, report_every=500)
        cmp = learned.compare(make_sim, 98, net, base=_lib.CF_PRECOND_LINE)
        print(f"held-out state: line patches {cmp.block_diagonal_iterations} iterations, learned-line "
              f"{cmp.learned_iterations} at weight {cmp.weight} (status {cmp.learned_status}), gain "
              f"{cmp.gain:.2f}; by weight {cmp.by_weight}; losses {losses}")
        assert losses[-1] < losses[0]
        assert cmp.use_learned == (cmp.learned_status == _lib.CF_OK and cmp.gain > 1.0)
        if cmp.gain < 1.0:
            pytest.xfail(f"the learned correction on top of the line patches loses on the held-out state: gain "
                         f"{cmp.gain:.2f} ({cmp.block_diagonal_iterations} -> {cmp.learned_iterations} iterations)")
        assert cmp.gain >= 1.0
