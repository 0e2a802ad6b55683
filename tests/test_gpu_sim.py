"""GPU parity of the device-resident implicit step through the C ABI.

Stages are compared with the FP64 oracle (oracle/implicit.py, the restatement
of mobility_solver.cpp and filament.cpp); whole runs are compared with the
reference's own generalised-force tables and with oracle trajectories.
Tolerances: FP64 stages 1e-10 relative; anything that contains the FP32 pair
mobility 1e-5 relative (the mobility contract); trajectories as stated below.
"""
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import implicit
from cufcm_fil_b200 import _lib, workloads
from cufcm_fil_b200.sim import WallCiliaSimulation, write_generalised_forces_run

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")


@pytest.fixture(scope="module")
def s_table():
    # Arclength table of the Fulford-Blake beat over one period from the oracle's bisection
    # (the reference's WRITE_GENERALISED_FORCES run writes the same table).
    _, _, sv = implicit.write_generalised_forces_run(1, tol=1e-3)
    return sv


def make_pair(nx, spacing, s_table, seed=0, **kw):
    F = nx * nx
    bases = workloads.lattice_bases(F, nx, spacing, 1.3)
    rng = np.random.default_rng(seed)
    phase0 = rng.uniform(0, 2 * np.pi, F)
    angle0 = rng.normal(0, 0.05, F)
    args = dict(nseg=20, seg_sep=2.6, dt=1 / 300, phase0=phase0, angle0=angle0, spring_factor=0.01,
                phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"], s_table=s_table)
    args.update(kw)
    tol = args.pop("gmres_tol", 1e-6)
    gpu = WallCiliaSimulation(bases=bases, gmres_tol=tol, **args)
    cpu = implicit.WallCilia(bases=bases, shape_sequence=1, gmres_tol=tol,
                             **{k: v for k, v in args.items() if k not in ("beat", "precond")})
    return gpu, cpu


def test_kinematics_rhs_match_oracle(s_table):
    gpu, cpu = make_pair(3, 40.0, s_table)
    with gpu:
        gpu.initial_guess(0)
        cpu.initial_guess(0)
        x, _ = gpu.segments()
        kp, ka = gpu.directions()
        np.testing.assert_allclose(x.reshape(-1, 3), cpu.x, rtol=0, atol=2e-5)   # float32 output
        np.testing.assert_allclose(kp, cpu.kp.ravel(), rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(ka, cpu.ka.ravel(), rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(gpu.arclengths(), cpu.s_values, rtol=0, atol=1e-12)
        rhs = gpu.assemble_rhs(0)
        np.testing.assert_allclose(rhs, cpu.assemble_rhs(), rtol=1e-11, atol=1e-6)


def test_bisection_arclengths_match_oracle():
    with WallCiliaSimulation(bases=[[0, 0, 1.3]], nseg=20, seg_sep=2.6, dynamic_phase=False,
                             dynamic_angle=False) as gpu:
        beat = oracle.beat.Beat(1, 20)
        for nt in range(300):
            gpu.initial_guess(nt)  # the phase advances by omega0*dt = 2 pi/300 per step after step 0
            if nt % 37 == 0:
                psi = 2 * math.pi * nt / 300
                np.testing.assert_allclose(gpu.arclengths()[0], beat.s_bisection(psi), atol=1e-9)


@pytest.mark.parametrize("dyn", [(True, True), (True, False), (False, True), (False, False)])
def test_preconditioner_and_saddle_product_match_oracle(s_table, dyn):
    gpu, cpu = make_pair(3, 40.0, s_table, dynamic_phase=dyn[0], dynamic_angle=dyn[1])
    with gpu:
        gpu.initial_guess(0)
        cpu.initial_guess(0)
        assert gpu.size == cpu.size
        rng = np.random.default_rng(11)
        for _ in range(2):
            v = rng.standard_normal(gpu.size)
            np.testing.assert_allclose(gpu.apply_preconditioner_new(v), cpu.precond(v), rtol=1e-10, atol=1e-10)
            got = gpu.system_matrix_mult_new(v)
            ref = cpu.matvec(v)
            assert oracle.rel_l2(got, ref) <= 1e-5


def test_write_generalised_forces_run_matches_reference_table():
    # One filament, prescribed phase speed, 300 steps: the reference's own generalised-force table
    # (written in FP32 with GMRES tolerance 1e-4) to 1e-4 relative L2.
    qp, qa = write_generalised_forces_run(_lib.CF_BEAT_FULFORD_BLAKE, nseg=20, seg_sep=2.6, steps=300, tol=1e-8)
    assert np.linalg.norm(qp - GOLD["fb_phase"]) / np.linalg.norm(GOLD["fb_phase"]) < 1e-4
    assert np.linalg.norm(qa - GOLD["fb_angle"]) / np.linalg.norm(GOLD["fb_angle"]) < 1e-4


def test_step_solution_satisfies_system_and_matches_oracle(s_table):
    gpu, cpu = make_pair(4, 20.0, s_table, seed=3)
    with gpu:
        res = gpu.step(0)
        it_cpu, rel_cpu = cpu.step(0)
        assert res.status == _lib.CF_OK and res.relative_residual <= 1e-6
        st = gpu.state()
        # the converged phase/angle rates agree with the oracle's FP64 GMRES to the solver tolerance
        np.testing.assert_allclose(st["phase_dot"], cpu.phase_dot, rtol=5e-5, atol=1e-5)
        np.testing.assert_allclose(st["angle_dot"], cpu.angle_dot, rtol=5e-5, atol=1e-5)
        # true FP64 residual of the GPU solution against the oracle operator
        _, fs = gpu.segments()
        sol = np.concatenate([fs.reshape(-1, 6)[:, :3].astype(np.float64).ravel(), st["phase_dot"], st["angle_dot"]])
        r = cpu.assemble_rhs() - cpu.matvec(sol)
        assert np.linalg.norm(r) / np.linalg.norm(cpu.assemble_rhs()) < 2e-5
        assert abs(res.iterations - it_cpu) <= max(3, 0.2 * it_cpu)


@pytest.mark.parametrize("spacing,steps,tip_tol", [(60.0, 90, 1e-3), (20.0, 10, 2e-3)])
def test_tip_trajectories_match_oracle(s_table, spacing, steps, tip_tol):
    # 16 cilia x 20 segments; tips after `steps` implicit steps at GMRES tolerance 1e-6.
    # At spacing 20 neighbouring cilia overlap and the dynamics are chaotic: the FP64 oracle run
    # with FP32 pair sums departs from the same run in FP64 by ~4e-4 L after 10 steps and by O(L)
    # after 40, so the dense case is compared over 10 steps only.
    # At spacing 60 the first 90 steps are well conditioned (a 1e-7 change of the initial phases
    # moves the oracle's tips by 2.5e-6 L by step 89); between steps ~90 and ~105 the saddle
    # system of this array is nearly singular and the same change grows to 1e-3 L (1e-2 L by
    # step 300), so later steps are fixed by the rounding of the sums, not by the physics.
    gpu, cpu = make_pair(4, spacing, s_table, seed=5)
    L = 2.6 * 19
    with gpu:
        worst = 0.0
        for nt in range(steps):
            gpu.step(nt)
            cpu.step(nt)
            if nt % 30 == 29 or nt == steps - 1:
                worst = max(worst, np.abs(gpu.tips() - cpu.tips()).max() / L)
        assert worst < tip_tol, worst


def test_async_steps_equal_sync_steps(s_table):
    g1, _ = make_pair(4, 20.0, s_table, seed=9)
    g2, _ = make_pair(4, 20.0, s_table, seed=9)
    with g1, g2:
        for nt in range(5):
            g1.step(nt)
            g2.step_async(nt)
        g2.last_solve()
        np.testing.assert_array_equal(g1.tips(), g2.tips())
        np.testing.assert_array_equal(g1.state()["phase"], g2.state()["phase"])


def test_zero_rhs_gives_zero_solution():
    # prescribed phase speed 0 and no dynamic unknowns: RHS = 0 -> lambda = 0 (mobility_solver.cpp:2222-2290)
    with WallCiliaSimulation(bases=[[0, 0, 1.3], [30, 0, 1.3]], dynamic_phase=False, dynamic_angle=False,
                             omega0=[0.0, 0.0]) as gpu:
        res = gpu.step(0)
        _, fs = gpu.segments()
        assert res.iterations == 0 and np.all(fs == 0.0)


def test_step_io_equals_separate_calls(s_table):
    gpu_a, _ = make_pair(3, 40.0, s_table, seed=8)
    gpu_b, _ = make_pair(3, 40.0, s_table, seed=8)
    with gpu_a, gpu_b:
        st = gpu_a.state()
        state = tuple(np.array(st[k]) for k in ("phase", "angle", "phase_dot", "angle_dot"))
        x = np.zeros(3 * gpu_a.n_seg_total, np.float32)
        f = np.zeros(6 * gpu_a.n_seg_total, np.float32)
        for nt in range(3):
            ra = gpu_a.step_io(nt, state_in=state, state_out=state, x_segs=x, f_segs=f)
            rb = gpu_b.step(nt)
            assert ra.iterations == rb.iterations and ra.status == rb.status
        sb = gpu_b.state()
        for arr, key in zip(state, ("phase", "angle", "phase_dot", "angle_dot")):
            np.testing.assert_array_equal(arr, sb[key])
        xb, fb = gpu_b.segments()
        np.testing.assert_array_equal(x, xb)
        np.testing.assert_array_equal(f, fb)


@pytest.mark.parametrize("precond", [_lib.CF_PRECOND_BLOCK_DIAG, _lib.CF_PRECOND_LINE])
def test_solve_on_given_rhs_matches_oracle(s_table, precond):
    # cf_sim_solve on a random RHS for the geometry of step 0, against the dense FP64 solve of the
    # oracle's operator (system_matrix_mult_new restated), twice (cold start, then the solution as the
    # guess).  The engine solves its own operator, whose pair sums are FP32: the FP64 residual of its
    # solution is bounded by the solver tolerance plus a backward error of the FP32 products,
    # |rhs - A x| <= tol |rhs| + c |A| |x| (c = 1e-8; the random RHS gives |x| ~ 200 |rhs|).
    gpu, cpu = make_pair(3, 30.0, s_table, seed=11, precond=precond)
    with gpu:
        gpu.initial_guess(0)
        cpu.initial_guess(0)
        n = cpu.size
        A = np.stack([cpu.matvec(e) for e in np.eye(n)], axis=1)
        rhs = np.random.default_rng(2).standard_normal(n)
        x_exact = np.linalg.solve(A, rhs)
        with pytest.raises(_lib.CufilError):
            gpu.solve_linear_system(rhs, tol=1e-6, max_iter=10_000)   # cap above the handle's
        x, res = gpu.solve_linear_system(rhs, tol=1e-6)
        assert res.status == _lib.CF_OK and res.relative_residual <= 1e-6
        bound = 1e-6 * np.linalg.norm(rhs) + 1e-8 * np.linalg.norm(np.abs(A) @ np.abs(x))
        assert np.linalg.norm(rhs - A @ x) <= bound
        assert np.linalg.norm(x - x_exact) / np.linalg.norm(x_exact) < 1e-3
        st = gpu.state()
        np.testing.assert_array_equal(st["phase_dot"], x[3 * cpu.nseg_total:3 * cpu.nseg_total + cpu.nfil])
        # The solution as the guess: kept unchanged when its residual meets the tolerance.  The
        # recomputed residual of x carries the FP32 product's rounding (~1e-5 of |rhs| here, as
        # |x| ~ 200 |rhs|), so the guess test uses 1e-4; at 1e-6 a few iterations restore it.
        x2, res2 = gpu.solve_linear_system(rhs, x0=x, tol=1e-4)
        assert res2.iterations == 0 and np.array_equal(x2, x)
        _, res4 = gpu.solve_linear_system(rhs, x0=x, tol=1e-6)
        assert res4.status == _lib.CF_OK and res4.iterations <= 10
        _, res3 = gpu.solve_linear_system(rhs, tol=1e-12, max_iter=3)
        assert res3.status == _lib.CF_NOT_CONVERGED and res3.iterations == 3


TIPS = np.load(Path(__file__).resolve().parent / "golden" / "ref_tips_16x16_80a.npz")
TIPS_TIGHT = np.load(Path(__file__).resolve().parent / "golden" / "ref_tips_16x16_80a_tight.npz")


def _run_300_steps(precond, tol, golden):
    nx = int(golden["nx"])
    F = nx * nx
    bases = workloads.lattice_bases(F, nx, float(golden["spacing"]), 1.3)
    with WallCiliaSimulation(bases=bases, nseg=20, seg_sep=2.6, dt=1 / 300, phase0=golden["phase0"],
                             angle0=golden["angle0"], spring_factor=0.01, phase_refs=GOLD["fb_phase"],
                             angle_refs=GOLD["fb_angle"], s_table=golden["s_table"], gmres_tol=tol,
                             precond=precond) as gpu:
        L = 2.6 * 19
        saved = list(golden["saved_steps"])
        worst_tip = worst_phase = 0.0
        for nt in range(int(golden["steps"])):
            res = gpu.step(nt)
            assert res.status == _lib.CF_OK and res.relative_residual <= tol
            if nt in saved:
                q = saved.index(nt)
                worst_tip = max(worst_tip, np.abs(gpu.tips() - golden["tips"][q]).max() / L)
                worst_phase = max(worst_phase, np.abs(gpu.state()["phase"] - golden["phase"][q]).max())
    return worst_tip, worst_phase


def test_300_steps_of_256_cilia_follow_the_reference_trajectory():
    # 256 cilia x 20 segments on a 16 x 16 lattice at 80a for 300 implicit steps (one beat period)
    # against the reference's own step code in FP64 at the same GMRES tolerance (1e-6) with the same
    # (block-diagonal) preconditioner (tests/golden/make_tip_golden.py).  At 80a no segments of
    # different cilia come within 19a of each other, so the saddle system stays well posed and the
    # trajectory is not chaotic: the engine takes the reference's Krylov path, and its FP32 pair
    # sums move the tips by at most TIP_TOL of the filament length over the whole period.
    TIP_TOL = 2e-4
    worst_tip, worst_phase = _run_300_steps(_lib.CF_PRECOND_BLOCK_DIAG, 1e-6, TIPS)
    print(f"256 cilia x 300 steps: worst tip error {worst_tip:.2e} L, worst phase error {worst_phase:.2e}")
    assert worst_tip < TIP_TOL and worst_phase < 2 * np.pi * TIP_TOL


def test_300_steps_with_line_patches_follow_the_converged_trajectory():
    # A relative residual of 1e-6 leaves the phase and angle rates of this saddle system accurate to
    # ~1e-3 only (the rate unknowns are weakly determined by the residual): at step 0 the reference's
    # block-diagonal GMRES at 1e-6 is 8.3e-3 off the exact rates, the line patches at 1e-6 1.8e-3, so
    # two preconditioners at 1e-6 follow trajectories ~1e-2 L apart after one period.  The line-patch
    # engine is therefore compared with the reference's trajectory at GMRES tolerance 1e-10
    # (make_tip_golden.py --tight), itself run at 1e-8.
    TIP_TOL = 2e-4
    worst_tip, worst_phase = _run_300_steps(_lib.CF_PRECOND_LINE, 1e-8, TIPS_TIGHT)
    print(f"line patches at 1e-8, 300 steps: worst tip error {worst_tip:.2e} L, worst phase error {worst_phase:.2e}")
    assert worst_tip < TIP_TOL and worst_phase < 2 * np.pi * TIP_TOL
