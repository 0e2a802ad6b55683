"""Drop-in for the reference's `cilia` executable, wall of prescribed cilia.

The reference's sweep drivers (pyfile/find_periodic/driver.py:92-104,
pyfile/bisection/driver.py) write input/globals.ini and an initial-condition
file, run ./bin/<exe> in the working directory and read
<simulation_dir><simulation_file>_true_states.dat back.  This module does the
same job on the engine: it reads the same inputs the reference reads
(globals.ini: cilia_sim_main.cu:59-91; the generalised-force tables and, when
present, the s-value table under input/forcing/: mobility_solver.cpp:45-107,
cilia_sim_main.cu:340-375; the initial condition: filament.cpp:310-340),
steps TOTAL_TIME_STEPS = sim_length * 300 + 1 implicit steps of DT =
period / 300, and appends the reference's data files every 10 steps
(cilia_sim_main.cu:624-718).  The wall build of the reference forces
NSWIM = 1 and NBLOB = 0 (cilia_sim_main.cu:96-99); features outside the
engine's path (FENE spring, force noise, frequency spread) are refused with an
error instead of being ignored.

  python -m cufcm_fil_b200.cilia [--ini input/globals.ini] [--tol 1e-4] [--precond line|block]

A driver keeps calling ./bin/<exe> after pointing it at this module, e.g. a
two-line shell script `exec python -m cufcm_fil_b200.cilia "$@"`.
"""
from __future__ import annotations

import argparse
import configparser
import ctypes
import math
import sys
from pathlib import Path

import numpy as np

from . import _lib, workloads

STEPS_PER_PERIOD = 300        # config.hpp: STEPS_PER_PERIOD
PLOT_FREQUENCY_IN_STEPS = 10  # STEPS_PER_PERIOD / SAVES_PER_PERIOD


def _forcing_name(kind: str, nseg: int, seg_sep: float) -> str:
    # filament.cpp:2300-2310 (Fulford-Blake beat): std::to_string of NSEG and SEG_SEP
    return f"input/forcing/fulford_and_blake_reference_{kind}_NSEG={nseg}_SEP={seg_sep:.6f}.dat"


def _read_vec(path: Path) -> np.ndarray:
    t = path.read_text().split()
    n = int(float(t[0]))
    return np.array([float(x) for x in t[1:1 + n]])


def read_ic(path, n_fil: int):
    """(header [2], phases [F], angles [F]) of an initial-condition file (cf_read_ic)."""
    h, p, a = np.zeros(2), np.zeros(n_fil), np.zeros(n_fil)
    _lib.call("cf_read_ic", str(path).encode(), int(n_fil), ctypes.c_void_p(h.ctypes.data),
              ctypes.c_void_p(p.ctypes.data), ctypes.c_void_p(a.ctypes.data))
    return h, p, a


def read_globals(ini: Path) -> dict:
    cp = configparser.ConfigParser()
    if not cp.read(ini):
        raise FileNotFoundError(f"{ini} not found")
    P, F = cp["Parameters"], cp["Filenames"]
    g = {k: float(P[k]) for k in ("nseg", "nfil", "seg_sep", "period", "sim_length", "spring_factor",
                                  "fil_x_dim", "fil_spacing")}
    for k in ("fene_model", "force_noise_mag", "omega_spread"):
        if float(P.get(k, "0")) != 0.0:
            raise ValueError(f"globals.ini: {k} = {P[k]} is not supported by this engine (only 0)")
    g["simulation_dir"] = F["simulation_dir"]
    g["simulation_file"] = F["simulation_file"]
    g["simulation_icstate_name"] = F.get("simulation_icstate_name", "input/psi.dat")
    return g


def run(ini="input/globals.ini", tol: float = 1e-4, precond: str = "line", device: int = 0, log=sys.stdout):
    """Runs one simulation as the reference's executable would; returns the output prefix."""
    from .sim import WallCiliaSimulation, arclength_table
    g = read_globals(Path(ini))
    nseg, nfil = int(g["nseg"]), int(g["nfil"])
    seg_sep, period = g["seg_sep"], g["period"]
    total = int(g["sim_length"] * STEPS_PER_PERIOD) + 1   # TOTAL_TIME_STEPS (cilia_sim_main.cu:125)
    dt = period / STEPS_PER_PERIOD
    prefix = g["simulation_dir"] + g["simulation_file"]
    Path(prefix).parent.mkdir(parents=True, exist_ok=True)
    phase_file = Path(_forcing_name("phase_generalised_forces", nseg, seg_sep))
    angle_file = Path(_forcing_name("angle_generalised_forces", nseg, seg_sep))
    for f in (phase_file, angle_file):
        if not f.exists():
            raise FileNotFoundError(f"required reference file {f} was not found (run the generalised-force pre-run)")
    s_file = Path(_forcing_name("s_values", nseg, seg_sep))
    if s_file.exists():
        t = s_file.read_text().split()
        rows, cols = int(float(t[0])), int(float(t[1]))
        s_table = np.array([float(x) for x in t[2:2 + rows * cols]]).reshape(rows, cols)
    else:  # the table the pre-run would write, by the same bisection
        s_table = arclength_table(nseg=nseg, seg_sep=seg_sep, steps=STEPS_PER_PERIOD)
    ic = Path(g["simulation_icstate_name"])
    if ic.exists():
        _, phase0, angle0 = read_ic(ic, nfil)
    else:  # filament.cpp:311-314: uniform random phases, zero angles
        print(f"No true_states file found: {ic}", file=log)
        phase0, angle0 = np.random.default_rng().uniform(0.0, 2.0 * math.pi, nfil), np.zeros(nfil)
    bases = workloads.lattice_bases(nfil, int(g["fil_x_dim"]), g["fil_spacing"], 0.5 * seg_sep)
    code = {"line": _lib.CF_PRECOND_LINE, "block": _lib.CF_PRECOND_BLOCK_DIAG}[precond]
    with WallCiliaSimulation(bases=bases, nseg=nseg, seg_sep=seg_sep, dt=dt, phase0=phase0, angle0=angle0,
                             spring_factor=g["spring_factor"], phase_refs=_read_vec(phase_file),
                             angle_refs=_read_vec(angle_file), s_table=s_table, gmres_tol=tol, precond=code,
                             device=device) as sim:
        sim.write_config(prefix, total)
        print(f"Simulating {nfil} filaments on an infinite no-slip wall, with each filament comprised of {nseg} "
              "segments.", file=log)
        for nt in range(total):
            res = sim.step(nt)
            if res.status == _lib.CF_NONFINITE:
                raise RuntimeError(f"step {nt + 1}: the linear solve met a non-finite value")
            if nt % PLOT_FREQUENCY_IN_STEPS == 0:
                sim.write_data(nt, period, prefix)
            print(f"Completed step {nt + 1}/{total} in {res.iterations} iterations of the linear system solver.",
                  file=log)
    return prefix


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cufcm_fil_b200.cilia")
    ap.add_argument("--ini", default="input/globals.ini")
    ap.add_argument("--tol", type=float, default=1e-4, help="GMRES relative tolerance (LINEAR_SYSTEM_TOL)")
    ap.add_argument("--precond", choices=["line", "block"], default="line")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    run(a.ini, a.tol, a.precond, a.device)


if __name__ == "__main__":
    main()
