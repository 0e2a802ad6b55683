"""The whole-step oracle against the reference's own step code, on the CPU.

oracle/_ref/ref_step_* are the reference's host sources (mobility_solver.cpp,
filament.cpp, swimmer.cpp, ...) compiled unmodified by oracle/ref_build.py and
driven by oracle/ref_step_harness.cu; in the FP64 variants the wall RPY
products come from the oracle's C restatement.  These tests pin the Python
restatement of the implicit step (oracle/implicit.py) -- RHS, block-diagonal
preconditioner, saddle product, GMRES, beat kinematics, dynamic phase and
angle coupling between filaments -- to the reference's own code, and show
where the model itself stops being well posed (overlapping segments).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import implicit, ref_step
from cufcm_fil_b200 import workloads

pytestmark = pytest.mark.skipif(not ref_step.available("step_dyn_f64") or not ref_step.available("step_wgf_f64"),
                                reason="reference step binaries not built (oracle/ref_build.py)")

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")
L = 2.6 * 19


@pytest.fixture(scope="module")
def wgf():
    return ref_step.wgf_tables(20, 2.6)


def test_reference_prerun_reproduces_its_shipped_tables(wgf):
    # The shipped tables were written by the reference's FP32 build at GMRES tolerance 1e-4;
    # this pre-run is the FP64 build at 1e-6.
    qp, qa, sv = wgf
    assert oracle.rel_l2(qp, GOLD["fb_phase"]) < 3e-5
    assert oracle.rel_l2(qa, GOLD["fb_angle"]) < 3e-5
    assert sv.shape == (300, 20) and np.all(np.diff(sv, axis=1) > 0)


def test_oracle_prerun_matches_reference_prerun(wgf):
    qp, qa, sv = wgf
    # The reference writes the s-value table with six significant digits (default stream
    # precision, filament.cpp:1136-1170); the oracle's bisection agrees to that rounding.
    oqp, oqa, osv = implicit.write_generalised_forces_run(1, tol=1e-6)
    assert np.abs(osv - sv).max() < 1e-6
    assert oracle.rel_l2(oqp, qp) < 1e-5 and oracle.rel_l2(oqa, qa) < 1e-5


def _pair(nx, spacing, seed, steps, s_table):
    F = nx * nx
    rng = np.random.default_rng(seed)
    phase0 = rng.uniform(0, 2 * np.pi, F)
    angle0 = rng.normal(0, 0.05, F)
    ref = ref_step.run(nfil=F, fil_x_dim=nx, spacing=spacing, phase0=phase0, angle0=angle0, steps=steps,
                       phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"], s_table=s_table)
    cpu = implicit.WallCilia(bases=workloads.lattice_bases(F, nx, spacing, 1.3), shape_sequence=1, nseg=20,
                             seg_sep=2.6, dt=1 / 300, phase0=phase0, angle0=angle0, spring_factor=0.01,
                             phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"], s_table=s_table,
                             gmres_tol=1e-6)
    return ref, cpu


@pytest.mark.parametrize("nx,spacing,steps", [(4, 60.0, 40), (3, 20.0, 8)])
def test_oracle_step_equals_reference_step(wgf, nx, spacing, steps):
    # Same lattice (the reference's rectangular seeding), same tables, same seeded phases:
    # the FP64 restatement follows the reference's own step to rounding, iteration counts included.
    ref, cpu = _pair(nx, spacing, 5, steps, wgf[2])
    for nt in range(steps):
        it, _ = cpu.step(nt)
        assert it == ref.iterations[nt]
        assert np.abs(cpu.tips() - ref.tips[nt]).max() / L < 1e-10
        np.testing.assert_allclose(cpu.phase_dot, ref.phase_dot[nt], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(cpu.angle_dot, ref.angle_dot[nt], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(cpu.angle, ref.angle[nt], rtol=0, atol=1e-12)


def test_overlapping_segments_break_definiteness(wgf):
    # At spacing 60a the beat (which sweeps -27a..35a along the beat direction) brings segments
    # of neighbouring cilia closer than 2a (they overlap) around step 80 of this seed, and the
    # wall RPY tensor, which like the reference has no overlap branch, is then indefinite: the
    # saddle system can become nearly singular.  Before the contact the tensor is positive definite.
    _, cpu = _pair(4, 60.0, 5, 1, wgf[2])
    dmins, eig = [], {}
    for nt in range(82):
        cpu.step(nt)
        X = cpu.x
        d = np.sqrt(((X[:, None, :] - X[None, :, :]) ** 2).sum(-1))
        fid = np.repeat(np.arange(cpu.nfil), cpu.nseg)
        d[fid[:, None] == fid[None, :]] = np.inf
        dmins.append(d.min())
        if nt in (10, 81):
            n = X.shape[0]
            M = np.zeros((3 * n, 3 * n))
            for c in range(3 * n):
                e = np.zeros(3 * n)
                e[c] = 1.0
                M[:, c] = cpu.mobility(e)
            eig[nt] = np.linalg.eigvalsh(0.5 * (M + M.T)).min()
    assert dmins[10] > 5.0 and eig[10] > 0.0
    assert dmins[81] < 1.0 and eig[81] < 0.0
