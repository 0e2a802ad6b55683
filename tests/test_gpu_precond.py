"""GPU tests of the line-patch block-Jacobi preconditioner (CF_PRECOND_LINE).

The patch inverses are formed on the device in FP32 by a blocked Gauss-Jordan
elimination; the oracle forms the same patches (oracle.implicit.line_patches)
and solves each patch block exactly in FP64.  Tolerance of the applied
preconditioner: 1e-3 relative L2 (FP32 assembly and inversion of blocks with
condition numbers up to ~1e3).  The GMRES solution is checked through the
system itself (the residual is always formed with the exact operator), and the
iteration count against the block-diagonal preconditioner on the same state.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import implicit
from cufcm_fil_b200 import _lib, workloads
from cufcm_fil_b200.sim import WallCiliaBatch, WallCiliaSimulation

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")


@pytest.fixture(scope="module")
def s_table():
    _, _, sv = implicit.write_generalised_forces_run(1, tol=1e-3)
    return sv


def make(n_fil, fil_x_dim, s_table, seed=0, precond=_lib.CF_PRECOND_LINE, line_patch=4, precond_refresh=0, **kw):
    bases = workloads.lattice_bases(n_fil, fil_x_dim, 20.0, 1.3)
    rng = np.random.default_rng(seed)
    args = dict(nseg=20, seg_sep=2.6, dt=1 / 300, phase0=rng.uniform(0, 2 * np.pi, n_fil),
                angle0=rng.normal(0, 0.05, n_fil), spring_factor=0.01, phase_refs=GOLD["fb_phase"],
                angle_refs=GOLD["fb_angle"], s_table=s_table)
    args.update(kw)
    gpu = WallCiliaSimulation(bases=bases, precond=precond, line_patch=line_patch, precond_refresh=precond_refresh,
                              **args)
    cpu = implicit.WallCilia(bases=bases, shape_sequence=1, **args)
    return gpu, cpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("geom", [(24, 4, 4), (32, 2, 16)])
@pytest.mark.parametrize("dyn", [(True, True), (True, False), (False, False)])
def test_patch_preconditioner_matches_oracle(s_table, dyn, geom):
    # (24, 4, 4): 4 x 6 lattice, lines of 6 filaments along y cut into patches of 3 (186 unknowns,
    # three pivot blocks, the last one partial); (32, 2, 16): two lines of 16 filaments, one patch
    # each (992 unknowns with both rates: 16 pivot blocks, the last 32 wide)
    n_fil, nx, lp = geom
    gpu, cpu = make(n_fil, nx, s_table, dynamic_phase=dyn[0], dynamic_angle=dyn[1], line_patch=lp)
    with gpu:
        gpu.initial_guess(0)
        cpu.initial_guess(0)
        v = np.random.default_rng(5).standard_normal(gpu.size)
        out = gpu.apply_preconditioner_new(v)
        ref = cpu.line_patch_precond(v, line_patch=lp)
        assert rel(out, ref) < 1e-3, rel(out, ref)
        # a patch inverse applied to its own block reproduces the input
        back = cpu.matvec(ref)
        fils = implicit.line_patches(cpu.bases, lp)[0]
        rows = cpu.patch_rows(fils)
        np.testing.assert_allclose(cpu.patch_block(fils) @ ref[rows], v[rows], rtol=1e-8, atol=1e-8)
        assert np.all(np.isfinite(back))


def true_relres(gpu, cpu):
    """FP64 residual of the GPU step solution against the oracle operator of the same state."""
    st = gpu.state()
    _, fs = gpu.segments()
    sol = np.concatenate([fs.reshape(-1, 6)[:, :3].astype(np.float64).ravel(), st["phase_dot"], st["angle_dot"]])
    rhs = cpu.assemble_rhs()
    return np.linalg.norm(rhs - cpu.matvec(sol)) / np.linalg.norm(rhs)


def test_line_step_solves_the_system_in_fewer_iterations(s_table):
    # Overlapping neighbours make this system nearly singular in a few rate directions, so two
    # solutions at relative residual 1e-6 may differ there; each is checked through the
    # oracle operator instead (FP32 pair sums: 2e-5, as for the block-diagonal step).
    for seed in (3, 4):
        gl, cpu = make(24, 4, s_table, seed=seed)
        gb, _ = make(24, 4, s_table, seed=seed, precond=_lib.CF_PRECOND_BLOCK_DIAG)
        with gl, gb:
            rl = gl.step(0)
            rb = gb.step(0)
            cpu.initial_guess(0)
            assert rl.status == _lib.CF_OK and rb.status == _lib.CF_OK
            assert rl.relative_residual <= 1e-6
            assert rl.iterations < rb.iterations, (rl.iterations, rb.iterations)
            assert true_relres(gl, cpu) < 2e-5
            assert true_relres(gb, cpu) < 2e-5


def test_line_patches_cut_iterations_on_colliding_cilia(s_table):
    # 16 x 16 lattice of spacing 20a with random phases: neighbours along the beat
    # direction overlap, the block-diagonal preconditioner needs >300 iterations
    gl, _ = make(256, 16, s_table, seed=100, line_patch=16)
    gb, _ = make(256, 16, s_table, seed=100, precond=_lib.CF_PRECOND_BLOCK_DIAG)
    with gl, gb:
        rl = gl.step(0)
        rb = gb.step(0)
        assert rl.status == _lib.CF_OK
        assert rl.iterations * 5 <= rb.iterations, (rl.iterations, rb.iterations)


def test_refresh_interval_keeps_convergence(s_table):
    # Inverses kept for 4 steps still precondition a converging solve (the residual is exact);
    # on colliding cilia a one-step-old inverse costs several times the iterations of a fresh one,
    # which is why the default refreshes every step.
    g1, _ = make(24, 4, s_table, seed=7, precond_refresh=1)
    g4, _ = make(24, 4, s_table, seed=7, precond_refresh=4)
    with g1, g4:
        for nt in range(6):
            r1 = g1.step(nt)
            r4 = g4.step(nt)
            assert r4.status == _lib.CF_OK and r4.relative_residual <= 1e-6
            if nt == 0:  # same state, same fresh inverses
                assert r4.iterations == r1.iterations


def test_nonfinite_state_reports_cleanly(s_table):
    gl, _ = make(24, 4, s_table, seed=2)
    with gl:
        ph = gl.state()["phase"]
        ph[3] = np.nan
        gl.set_state(phase=ph)
        gl.step_async(0)
        with pytest.raises(_lib.CufilError) as err:
            gl.last_solve()
        assert err.value.code == _lib.CF_NONFINITE


def test_batch_with_patches_matches_single_runs(s_table):
    specs = []
    for n, nx, seed in ((6, 2, 1), (12, 3, 2), (8, 2, 3)):
        rng = np.random.default_rng(seed)
        specs.append(dict(bases=workloads.lattice_bases(n, nx, 20.0, 1.3), phase0=rng.uniform(0, 2 * np.pi, n),
                          angle0=rng.normal(0, 0.05, n)))
    shared = dict(nseg=20, seg_sep=2.6, dt=1 / 300, spring_factor=0.01, phase_refs=GOLD["fb_phase"],
                  angle_refs=GOLD["fb_angle"], s_table=s_table, precond=_lib.CF_PRECOND_LINE, line_patch=4)
    singles = []
    for sp in specs:
        with WallCiliaSimulation(**shared, **sp) as s:
            its = [s.step(nt).iterations for nt in range(2)]
            singles.append((its, s.state()))
    with WallCiliaBatch(specs, **shared) as bt:
        for nt in range(2):
            it, _, rc = bt.step(nt)
            assert rc == _lib.CF_OK
            for b in range(len(specs)):
                assert it[b] == singles[b][0][nt]
        st = bt.state()
    for b in range(len(specs)):
        np.testing.assert_array_equal(st[b]["phase_dot"], singles[b][1]["phase_dot"])


def test_checkpoint_restore_repeats_the_trajectory(s_table):
    # Colliding cilia: the dynamics amplify any difference in the warm start, so a restore that
    # missed part of the state (the constraint forces seed the next GMRES) would change the iterations.
    gl, _ = make(24, 4, s_table, seed=11)
    with gl:
        for nt in range(2):
            gl.step(nt)
        ck = gl.checkpoint()
        first = [gl.step(nt).iterations for nt in range(2, 6)]
        end = gl.checkpoint()
        gl.step(6)  # move away, then come back
        gl.restore(ck)
        again = [gl.step(nt).iterations for nt in range(2, 6)]
        assert again == first
        back = gl.checkpoint()
        for key in ("phase", "angle", "phase_dot", "angle_dot", "solution"):
            np.testing.assert_array_equal(back[key], end[key])
