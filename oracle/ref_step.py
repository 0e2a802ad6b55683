"""Runs the reference's own prescribed-cilia step through oracle/_ref/ref_step_* (test infrastructure only).

The binaries are built by oracle/ref_build.py from the reference's host sources
(mobility_solver.cpp, filament.cpp, swimmer.cpp, ...) and ref_step_harness.cu;
see that file for what each variant links.  Each run happens in a scratch
directory laid out as the reference expects it (input/forcing/ for the
generalised-force and s-value tables, the initial-condition file in the
reference's psi.dat format: two header numbers, then the phases, then the
angles -- filament.cpp:310-340).

  wgf_tables(nseg, seg_sep)  the WRITE_GENERALISED_FORCES pre-run
                             (cilia_sim_main.cu:318-338, 420-440)
  run(...)                   a dynamic run of a rectangular wall lattice
                             (swimmer.cpp:113-185 seeding), per-step records
"""
from __future__ import annotations

import subprocess
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"


def binary(variant: str) -> Path:
    return REF / f"ref_{variant}"


def available(variant: str = "step_dyn_f64") -> bool:
    return binary(variant).exists()


def _tag(nseg: int, seg_sep: float) -> str:
    # filament.cpp:2300-2310: "NSEG=" + std::to_string(NSEG) + "_SEP=" + std::to_string(SEG_SEP)
    return f"NSEG={nseg}_SEP={seg_sep:.6f}.dat"


def _forcing_name(kind: str, nseg: int, seg_sep: float) -> str:
    return f"fulford_and_blake_reference_{kind}_{_tag(nseg, seg_sep)}"


def _write_vec(path: Path, v) -> None:
    v = np.asarray(v, float).ravel()
    path.write_text(f"{v.size} " + " ".join(repr(float(x)) for x in v))


def _read_vec(path: Path) -> np.ndarray:
    t = path.read_text().split()
    n = int(float(t[0]))
    return np.array([float(x) for x in t[1:1 + n]])


def wgf_tables(nseg: int = 20, seg_sep: float = 2.6, timeout: float = 600.0):
    """The reference's pre-run: returns (phase forces [300], angle forces [300], s-values [300, nseg])."""
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        (d / "input" / "forcing").mkdir(parents=True)
        subprocess.run([str(binary("step_wgf_f64")), "wgf", str(nseg), repr(float(seg_sep)), "out.bin"], cwd=d,
                       check=True, capture_output=True, timeout=timeout)
        f = d / "input" / "forcing"
        qp = _read_vec(f / _forcing_name("phase_generalised_forces", nseg, seg_sep))
        qa = _read_vec(f / _forcing_name("angle_generalised_forces", nseg, seg_sep))
        t = (f / _forcing_name("s_values", nseg, seg_sep)).read_text().split()
        rows, cols = int(float(t[0])), int(float(t[1]))
        sv = np.array([float(x) for x in t[2:2 + rows * cols]]).reshape(rows, cols)
    return qp, qa, sv


@dataclass
class RefRun:
    iterations: np.ndarray   # [steps] GMRES iterations (solve_linear_system's return value)
    seconds: np.ndarray      # [steps] host wall time of each step
    phase: np.ndarray        # [steps, F]
    angle: np.ndarray
    phase_dot: np.ndarray
    angle_dot: np.ndarray
    tips: np.ndarray         # [steps, F, 3] last segment of each filament
    files: dict | None = None  # data file suffix -> text, when run(write=True)


def run(*, nfil: int, fil_x_dim: int, spacing: float, phase0, angle0, steps: int, phase_refs, angle_refs,
        s_table, nseg: int = 20, seg_sep: float = 2.6, spring_factor: float = 0.01,
        variant: str = "step_dyn_f64", timeout: float = 3600.0, budget: float | None = None,
        write: bool = False) -> RefRun:
    """Dynamic run of the reference's step on an nfil lattice (fil_x_dim columns, spacing in radii).
    With `budget` (seconds) the run is stopped after that time and the steps finished so far are returned."""
    F = int(nfil)
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        f = d / "input" / "forcing"
        f.mkdir(parents=True)
        _write_vec(f / _forcing_name("phase_generalised_forces", nseg, seg_sep), phase_refs)
        _write_vec(f / _forcing_name("angle_generalised_forces", nseg, seg_sep), angle_refs)
        s = np.asarray(s_table, float)
        (f / _forcing_name("s_values", nseg, seg_sep)).write_text(
            f"{s.shape[0]} {s.shape[1]} " + " ".join(repr(float(x)) for x in s.ravel()))
        ic = np.concatenate([np.asarray(phase0, float), np.asarray(angle0, float)])
        (d / "psi.dat").write_text("0 0 " + " ".join(repr(float(x)) for x in ic))
        cmd = [str(binary(variant)), "run", str(nseg), str(F), str(int(fil_x_dim)), repr(float(spacing)),
               repr(float(seg_sep)), repr(float(spring_factor)), str(int(steps)), "psi.dat", "out.bin"]
        if write:
            cmd.append("write")
        if budget is None:
            subprocess.run(cmd, cwd=d, check=True, capture_output=True, timeout=timeout)
        else:
            try:
                subprocess.run(cmd, cwd=d, check=True, capture_output=True, timeout=budget)
            except subprocess.TimeoutExpired:
                pass  # the records of the finished steps are flushed one by one
        width = 2 + 7 * F
        raw = np.fromfile(d / "out.bin") if (d / "out.bin").exists() else np.zeros(0)
        rec = raw[:raw.size // width * width].reshape(-1, width)
        files = None
        if write:
            files = {p.name[len("ref_step"):]: p.read_text() for p in d.glob("ref_step_*.dat")}
    return RefRun(files=files, iterations=rec[:, 0].astype(int), seconds=rec[:, 1], phase=rec[:, 2:2 + F],
                  angle=rec[:, 2 + F:2 + 2 * F], phase_dot=rec[:, 2 + 2 * F:2 + 3 * F],
                  angle_dot=rec[:, 2 + 3 * F:2 + 4 * F], tips=rec[:, 2 + 4 * F:].reshape(-1, F, 3))


@dataclass
class RefBodyRun(RefRun):
    body_x: np.ndarray | None = None   # [steps, 3] body centre used in the step
    body_q: np.ndarray | None = None   # [steps, 4] body orientation (scalar first)
    body_v: np.ndarray | None = None   # [steps, 6] body velocity and angular velocity solved for


def _unit_sphere_frames(normals):
    """Seeding records of the reference (positions on the unit-length sphere of radius 1/2, polar and
    azimuthal directions, normals) for the given outward unit normals."""
    n = np.asarray(normals, float).reshape(-1, 3)
    pos = 0.5 * n
    ez = np.array([0.0, 0.0, 1.0])
    azi = np.cross(ez, n)
    nrm = np.linalg.norm(azi, axis=1)
    azi[nrm < 1e-12] = [1.0, 0.0, 0.0]
    azi /= np.linalg.norm(azi, axis=1)[:, None]
    polar = np.cross(azi, n)
    return pos, polar, azi, n


def _write_seeds(d: Path, count: int, normals) -> None:
    pos, polar, azi, n = _unit_sphere_frames(normals)
    stem = d / "input" / "fourier_modes" / f"sphere{count}"
    stem.parent.mkdir(parents=True, exist_ok=True)
    for ext, arr in (("seed", pos), ("polar_dir", polar), ("azi_dir", azi), ("normal", n)):
        stem.with_suffix("." + ext).write_text(" ".join(repr(float(v)) for v in arr.ravel()) + "\n")


def run_body(*, fil_normals, blob_normals, ar: float, phase0, angle0, steps: int, phase_refs, angle_refs, s_table,
             nseg: int = 20, seg_sep: float = 2.6, spring_factor: float = 0.01, timeout: float = 3600.0) -> RefBodyRun:
    """Dynamic run of the reference's step for one free spherical body (diameter ar * filament length) with
    filaments along `fil_normals` and blobs along `blob_normals` (unit vectors; the reference reads them as its
    seeding files, swimmer.cpp:310-345, rigid_body.cpp:330-380)."""
    fil_normals = np.asarray(fil_normals, float).reshape(-1, 3)
    blob_normals = np.asarray(blob_normals, float).reshape(-1, 3)
    F, B = fil_normals.shape[0], blob_normals.shape[0]
    if F == B:
        raise ValueError("the reference names its seeding files by count: use different filament and blob counts")
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        f = d / "input" / "forcing"
        f.mkdir(parents=True)
        _write_vec(f / _forcing_name("phase_generalised_forces", nseg, seg_sep), phase_refs)
        _write_vec(f / _forcing_name("angle_generalised_forces", nseg, seg_sep), angle_refs)
        s = np.asarray(s_table, float)
        (f / _forcing_name("s_values", nseg, seg_sep)).write_text(
            f"{s.shape[0]} {s.shape[1]} " + " ".join(repr(float(x)) for x in s.ravel()))
        _write_seeds(d, F, fil_normals)
        _write_seeds(d, B, blob_normals)
        ic = np.concatenate([np.asarray(phase0, float), np.asarray(angle0, float)])
        (d / "psi.dat").write_text("0 0 " + " ".join(repr(float(x)) for x in ic))
        cmd = [str(binary("step_body_f64")), "run", str(nseg), str(F), str(B), repr(float(ar)), repr(float(seg_sep)),
               repr(float(spring_factor)), str(int(steps)), "psi.dat", "out.bin"]
        subprocess.run(cmd, cwd=d, check=True, capture_output=True, timeout=timeout)
        width = 2 + 7 * F + 13
        raw = np.fromfile(d / "out.bin")
        rec = raw[:raw.size // width * width].reshape(-1, width)
    o = 2 + 7 * F
    return RefBodyRun(iterations=rec[:, 0].astype(int), seconds=rec[:, 1], phase=rec[:, 2:2 + F],
                      angle=rec[:, 2 + F:2 + 2 * F], phase_dot=rec[:, 2 + 2 * F:2 + 3 * F],
                      angle_dot=rec[:, 2 + 3 * F:2 + 4 * F], tips=rec[:, 2 + 4 * F:o].reshape(-1, F, 3),
                      body_x=rec[:, o:o + 3], body_q=rec[:, o + 3:o + 7], body_v=rec[:, o + 7:o + 13])



@dataclass
class RefElasticRun:
    iterations: np.ndarray   # [steps] Broyden iterations
    seconds: np.ndarray      # [steps]
    x: np.ndarray            # [steps, N, 3] segment positions after each step


def run_elastic(*, nfil: int, fil_x_dim: int, spacing: float, steps: int, nseg: int = 20, seg_sep: float = 2.6,
                period: float = 36.3833, timeout: float = 3600.0) -> RefElasticRun:
    """The reference's own step for instability-driven elastic cilia on a wall lattice (CILIA_TYPE 0,
    CILIA_IC_TYPE 0, FP64), run by ref_elastic_harness.cu; DT = period / 300."""
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        cmd = [str(binary("elastic_f64")), "run", str(nseg), str(int(nfil)), str(int(fil_x_dim)), repr(float(spacing)),
               repr(float(seg_sep)), repr(float(period)), str(int(steps)), "out.bin"]
        subprocess.run(cmd, cwd=d, check=True, capture_output=True, timeout=timeout)
        N = int(nfil) * nseg
        raw = np.fromfile(d / "out.bin")
        rec = raw[:raw.size // (2 + 3 * N) * (2 + 3 * N)].reshape(-1, 2 + 3 * N)
    return RefElasticRun(iterations=rec[:, 0].astype(int), seconds=rec[:, 1], x=rec[:, 2:].reshape(-1, N, 3))


def elastic_jacobian(*, nseg: int = 20, seg_sep: float = 2.6, period: float = 36.3833):
    """(inverse approximate Jacobian [6 nseg, 6 nseg], residual [6 nseg]) of one elastic filament at the
    first evaluation of step 0, from the reference's own invert_approx_jacobian."""
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        cmd = [str(binary("elastic_f64")), "jac", str(nseg), repr(float(seg_sep)), repr(float(period)), "out.bin"]
        subprocess.run(cmd, cwd=d, check=True, capture_output=True, timeout=600)
        raw = np.fromfile(d / "out.bin")
    n = 6 * nseg
    return raw[:n * n].reshape(n, n), raw[n * n:n * n + n]
