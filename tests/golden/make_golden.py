"""Writes tests/golden/reference_forcing_nseg20_sep2.6.npz from the reference's own tables.

Source (read as text): racksa/CUFCM_FIL input/forcing/
  fulford_and_blake_reference_{phase,angle}_generalised_forces_NSEG=20_SEP=2.600000.dat
  fulford_and_blake_original_reference_{phase,angle}_generalised_forces_NSEG=20_SEP=2.600000.dat
  fulford_and_blake_original_reference_s_values_NSEG=20_SEP=2.600000.dat
These are outputs of the reference's WRITE_GENERALISED_FORCES run (a single
prescribed filament above the wall, 300 steps over one period; written by
cilia_sim_main.cu:318-338,420-440 and filament.cpp:1122-1180), so they pin
the beat kinematics, the arclength bisection, the wall RPY mobility and the
linear solve of that run.  Format: "count v_1 ... v_count" for the forces,
"steps nseg s_1 ... s_(steps*nseg)" for the arclength table.

Run: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_forcing_nseg20_sep2.6.npz"


def read_vec(p):
    vals = p.read_text().split()
    n = int(float(vals[0]))
    v = np.array([float(x) for x in vals[1:1 + n]])
    assert v.size == n
    return v


def read_table(p):
    vals = p.read_text().split()
    rows, cols = int(float(vals[0])), int(float(vals[1]))
    t = np.array([float(x) for x in vals[2:2 + rows * cols]]).reshape(rows, cols)
    return t


def main(root):
    d = Path(root) / "input" / "forcing"
    tag = "NSEG=20_SEP=2.600000.dat"
    arrays = {
        "fb_phase": read_vec(d / f"fulford_and_blake_reference_phase_generalised_forces_{tag}"),
        "fb_angle": read_vec(d / f"fulford_and_blake_reference_angle_generalised_forces_{tag}"),
        "fbo_phase": read_vec(d / f"fulford_and_blake_original_reference_phase_generalised_forces_{tag}"),
        "fbo_angle": read_vec(d / f"fulford_and_blake_original_reference_angle_generalised_forces_{tag}"),
        "fbo_s_values": read_table(d / f"fulford_and_blake_original_reference_s_values_{tag}"),
    }
    np.savez_compressed(OUT, **arrays)
    print(OUT, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
    main(sys.argv[1])
