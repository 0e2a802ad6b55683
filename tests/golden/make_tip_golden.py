"""Writes tests/golden/ref_tips_16x16_80a.npz: a 300-step trajectory of the reference's own step.

The reference's prescribed-cilia host code (mobility_solver.cpp, filament.cpp,
swimmer.cpp, ... built with FIL_USE_DOUBLE_PRECISION true and LINEAR_SYSTEM_TOL
1e-6 by oracle/ref_build.py, driven by oracle/ref_step_harness.cu, wall RPY
products by the FP64 oracle) runs 256 Fulford-Blake cilia x 20 segments on a
16 x 16 wall lattice at spacing 80a (SEP 2.6, spring factor 0.01, dt = T/300)
for 300 steps, from phases U(0, 2 pi) and angles N(0, 0.05) of seed 80.  At 80a
no two segments of different cilia come closer than ~19a over the 300 steps
(the beat sweeps -27a..35a along the beat direction), so the saddle system stays
well posed.  The generalised-force tables are the reference's shipped ones
(reference_forcing_nseg20_sep2.6.npz); the s-value table is the one the
reference's own WRITE_GENERALISED_FORCES pre-run writes (stored here too, the
reference tree does not ship it for this beat).

With --tight the reference's GMRES tolerance is 1e-10 (variant step_dyn_f64_tight) and the
output is ref_tips_16x16_80a_tight.npz: the trajectory with near-exact linear solves, against
which solvers whose iterates differ from the reference's (other preconditioners) are compared.

Run: python tests/golden/make_tip_golden.py [--tight]   (needs the oracle/_ref binaries; ~10 min on 8 cores)
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle import ref_step  # noqa: E402

TIGHT = "--tight" in sys.argv
OUT = HERE / ("ref_tips_16x16_80a_tight.npz" if TIGHT else "ref_tips_16x16_80a.npz")
NX, SPACING, STEPS, SEED = 16, 80.0, 300, 80
SAVE = np.array(sorted(set(range(0, STEPS, 25)) | {STEPS - 1}))


def main():
    gold = np.load(HERE / "reference_forcing_nseg20_sep2.6.npz")
    qp, qa, s_table = ref_step.wgf_tables(20, 2.6)
    F = NX * NX
    rng = np.random.default_rng(SEED)
    phase0 = rng.uniform(0, 2 * np.pi, F)
    angle0 = rng.normal(0, 0.05, F)
    r = ref_step.run(nfil=F, fil_x_dim=NX, spacing=SPACING, phase0=phase0, angle0=angle0, steps=STEPS,
                     phase_refs=gold["fb_phase"], angle_refs=gold["fb_angle"], s_table=s_table,
                     variant="step_dyn_f64_tight" if TIGHT else "step_dyn_f64")
    np.savez_compressed(OUT, nx=NX, spacing=SPACING, steps=STEPS, seed=SEED, phase0=phase0, angle0=angle0,
                        gmres_tol=1e-10 if TIGHT else 1e-6,
                        s_table=s_table, wgf_phase=qp, wgf_angle=qa, saved_steps=SAVE,
                        tips=r.tips[SAVE], phase=r.phase[SAVE], angle=r.angle[SAVE],
                        phase_dot=r.phase_dot[SAVE], angle_dot=r.angle_dot[SAVE], iterations=r.iterations)
    print(OUT, "iterations per step: mean %.2f max %d" % (r.iterations.mean(), r.iterations.max()),
          "seconds per step %.2f" % r.seconds.mean())


if __name__ == "__main__":
    main()
