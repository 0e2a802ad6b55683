"""Imports the reference's generalised-force tables into fulford_blake_nseg20_sep2.6.npz.

The dynamic prescribed-cilia step needs the reference generalised phase and
angle forces over one beat (the reference reads them from
input/forcing/fulford_and_blake_reference_{phase,angle}_generalised_forces_NSEG=20_SEP=2.600000.dat,
mobility_solver.cpp:45-107).  This script converts those two text files
(format: count, then the values) into the package's input deck; it needs the
reference tree and is run once, by hand.

Run: python cufcm_fil_b200/data/import_reference_forcing.py [reference_root]
"""
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "fulford_blake_nseg20_sep2.6.npz"


def read_vec(p):
    vals = Path(p).read_text().split()
    n = int(float(vals[0]))
    return np.array([float(x) for x in vals[1:1 + n]])


def main(root="/root/reference"):
    d = Path(root) / "input" / "forcing"
    tag = "NSEG=20_SEP=2.600000.dat"
    np.savez_compressed(OUT, phase=read_vec(d / f"fulford_and_blake_reference_phase_generalised_forces_{tag}"),
                        angle=read_vec(d / f"fulford_and_blake_reference_angle_generalised_forces_{tag}"))
    print(OUT)


if __name__ == "__main__":
    main(*sys.argv[1:])
