"""Writes tests/golden/ref_elastic_2x2_80a.npz: the reference's own elastic-filament step.

The reference's host step code for instability-driven elastic cilia on a wall
(CILIA_TYPE 0, CILIA_IC_TYPE 0: a step-0 perturbation 0.01 F_end e_x on segment
4; mobility_solver.cpp, filament.cpp, swimmer.cpp, segment.cpp,
broyden_solver.cpp, ... built with FIL_USE_DOUBLE_PRECISION true by
oracle/ref_build.py, driven by oracle/ref_elastic_harness.cu, 6x6 wall RPY by
the FP64 oracle, barrier forces restated there) runs 4 filaments x 20 segments
on a 2 x 2 wall lattice at spacing 80a with SEP 2.6, DIMENSIONLESS_FORCE 220,
KB = KT = 1800 and DT = 36.3833/300, for 300 steps; the follower force buckles
the filaments and they start to beat within the run.  Stored: the Broyden
iterations of every step and the segment positions every 10 steps; and, for one
filament, the inverse approximate Jacobian and the residual of the first
evaluation of step 0 (the reference's invert_approx_jacobian).

Also writes tests/golden/ref_elastic_2x2_2p1a.npz: the same 2 x 2 lattice at spacing 2.1a for 20 steps, where
the bases of neighbouring cilia are closer than the barrier range 1.1 (a_i + a_j) = 2.2a, so the segment-segment
barrier forces act from the first evaluation; positions and Broyden iterations of every step.

Also writes tests/golden/ref_elastic_jinv_probes.npz: for one filament of 14, 20 and 24 segments, the reference's
inverse approximate Jacobian (first evaluation of step 0) times four seeded normal columns
(numpy default_rng(5)), and its Frobenius norm.  These cover each block size class of the device inversion.

Run: python tests/golden/make_elastic_golden.py   (needs the oracle/_ref binaries; a few seconds)
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle import ref_step  # noqa: E402

OUT = HERE / "ref_elastic_2x2_80a.npz"
OUT_CLOSE = HERE / "ref_elastic_2x2_2p1a.npz"
NX, SPACING, STEPS, PERIOD, EVERY = 2, 80.0, 300, 36.3833, 10
CLOSE_SPACING, CLOSE_STEPS = 2.1, 20
OUT_PROBES = HERE / "ref_elastic_jinv_probes.npz"
PROBE_NSEG = (14, 20, 24)


def write_probes():
    out = {}
    for ns in PROBE_NSEG:
        jinv, _ = ref_step.elastic_jacobian(nseg=ns, period=PERIOD)
        v = np.random.default_rng(5).standard_normal((6 * ns, 4))
        out[f"p{ns}"] = jinv @ v
        out[f"norm{ns}"] = np.linalg.norm(jinv)
    np.savez_compressed(OUT_PROBES, nseg=np.array(PROBE_NSEG), period=PERIOD, **out)
    print(OUT_PROBES)


def main():
    jinv, err0 = ref_step.elastic_jacobian(period=PERIOD)
    r = ref_step.run_elastic(nfil=NX * NX, fil_x_dim=NX, spacing=SPACING, steps=STEPS, period=PERIOD)
    saved = np.arange(0, STEPS, EVERY)
    np.savez_compressed(OUT, nx=NX, spacing=SPACING, steps=STEPS, period=PERIOD, saved_steps=saved,
                        x=r.x[saved], iterations=r.iterations, jinv0=jinv, err0=err0)
    print(OUT, "Broyden iterations per step: mean %.2f max %d" % (r.iterations.mean(), r.iterations.max()))
    c = ref_step.run_elastic(nfil=NX * NX, fil_x_dim=NX, spacing=CLOSE_SPACING, steps=CLOSE_STEPS, period=PERIOD)
    np.savez_compressed(OUT_CLOSE, nx=NX, spacing=CLOSE_SPACING, steps=CLOSE_STEPS, period=PERIOD, x=c.x,
                        iterations=c.iterations)
    print(OUT_CLOSE, "Broyden iterations per step:", c.iterations.tolist())
    write_probes()


if __name__ == "__main__":
    main()
