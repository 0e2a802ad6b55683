"""Writes tests/golden/ref_swim_12fil_642blob.npz: a 300-step trajectory of the reference's own free swimmer.

The reference's host step code for prescribed cilia on a free rigid body
(mobility_solver.cpp, filament.cpp, swimmer.cpp, rigid_body.cpp, ... built with
BODY_OR_SURFACE_TYPE 2, BODY_VELOCITY_TYPE 0, FIL_USE_DOUBLE_PRECISION true and
LINEAR_SYSTEM_TOL 1e-6 by oracle/ref_build.py, driven by
oracle/ref_step_harness.cu, unbounded RPY products over segments and blobs by
the FP64 oracle) runs 12 Fulford-Blake cilia x 20 segments on a sphere of
diameter 3 filament lengths (AR 3, radius 74.1a) represented by 642 blobs, for
300 steps (one beat period at dt = T/300), from phases U(0, 2 pi) and angles
N(0, 0.05) of seed 12.  Filament and blob directions are Fibonacci lattices on
the sphere (cufcm_fil_b200.swim.fibonacci_normals, offsets 0.5 and 0.3), written
as the reference's seeding files.  The bases lie ~79a apart, so cilia never
overlap and the system stays well posed.  Tables as in make_tip_golden.py.

Run: python tests/golden/make_swim_golden.py   (needs the oracle/_ref binaries; a few seconds)
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle import ref_step  # noqa: E402
from cufcm_fil_b200.swim import fibonacci_normals  # noqa: E402

OUT = HERE / "ref_swim_12fil_642blob.npz"
F, B, AR, STEPS, SEED = 12, 642, 3.0, 300, 12


def main():
    gold = np.load(HERE / "reference_forcing_nseg20_sep2.6.npz")
    _, _, s_table = ref_step.wgf_tables(20, 2.6)
    rng = np.random.default_rng(SEED)
    phase0 = rng.uniform(0, 2 * np.pi, F)
    angle0 = rng.normal(0, 0.05, F)
    fn, bn = fibonacci_normals(F), fibonacci_normals(B, 0.3)
    r = ref_step.run_body(fil_normals=fn, blob_normals=bn, ar=AR, phase0=phase0, angle0=angle0, steps=STEPS,
                          phase_refs=gold["fb_phase"], angle_refs=gold["fb_angle"], s_table=s_table)
    np.savez_compressed(OUT, n_fil=F, n_blob=B, ar=AR, steps=STEPS, seed=SEED, fil_normals=fn, blob_normals=bn,
                        phase0=phase0, angle0=angle0, s_table=s_table, phase=r.phase, angle=r.angle,
                        phase_dot=r.phase_dot, angle_dot=r.angle_dot, tips=r.tips, body_x=r.body_x,
                        body_q=r.body_q, body_v=r.body_v, iterations=r.iterations)
    print(OUT, "iterations per step: mean %.2f max %d" % (r.iterations.mean(), r.iterations.max()),
          "body displacement over the run", r.body_x[-1] - r.body_x[0])


if __name__ == "__main__":
    main()
