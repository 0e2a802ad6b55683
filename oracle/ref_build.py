"""Recipe that compiles the REFERENCE's own RPY kernels into oracle/_ref/ (test infrastructure).

The reference's ``src/cilia/cuda_functions.cu`` is compiled in place from the
reference tree (``/root/reference`` in the build container) for sm_100a,
together with ``ref_rpy_wrapper.cu`` which adds plain C launchers.  The
reference selects its physics with compile-time switches in ``config.hpp``;
for each variant this recipe writes a configuration header into
``oracle/_ref/`` by editing those switches in the reference's config.hpp, and
pre-includes it (``-include``) so that the reference's own ``config.hpp``
include guard turns the original into a no-op.  Outputs (headers, objects,
``libref_rpy_<variant>.so``) go only to ``oracle/_ref/``, which git ignores;
the built libraries travel with the tree so GPU tests can run them where the
reference sources are absent.

It also builds the reference's cuFCM solver (src/cufcm/*.cu, float, translation
only as configured) with ref_fcm_wrapper.cu into oracle/_ref/libref_fcm.so.

Variants (switches of config.hpp):
  wall3  CILIA_TYPE 3 (prescribed), BODY_OR_SURFACE_TYPE 0 (wall)  -- as mounted
  wall6  CILIA_TYPE 0 (6-dof segments), BODY_OR_SURFACE_TYPE 0
  free3  CILIA_TYPE 3, BODY_OR_SURFACE_TYPE 2 (unbounded)
  free6  CILIA_TYPE 0, BODY_OR_SURFACE_TYPE 2
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# The reference tree: set by the caller (set_reference_root) or the
# CUFIL_REFERENCE_ROOT environment variable; without it nothing is built.
REF_ROOT = Path(os.environ["CUFIL_REFERENCE_ROOT"]) if os.environ.get("CUFIL_REFERENCE_ROOT") else None


def set_reference_root(path) -> None:
    global REF_ROOT
    REF_ROOT = Path(path) if path else None
WRAPPER = HERE / "ref_rpy_wrapper.cu"

VARIANTS = {
    "wall3": {"CILIA_TYPE": "3", "BODY_OR_SURFACE_TYPE": "0"},
    "wall6": {"CILIA_TYPE": "0", "BODY_OR_SURFACE_TYPE": "0"},
    "free3": {"CILIA_TYPE": "3", "BODY_OR_SURFACE_TYPE": "2"},
    "free6": {"CILIA_TYPE": "0", "BODY_OR_SURFACE_TYPE": "2"},
}


def lib_path(variant: str) -> Path:
    return OUT / f"libref_rpy_{variant}.so"


def _config_text(switches: dict[str, str]) -> str:
    text = (REF_ROOT / "config.hpp").read_text()
    for key, val in switches.items():
        pat = re.compile(rf"^#define {key} \S+", re.M)
        if not pat.search(text):
            raise RuntimeError(f"switch {key} not found in the reference config.hpp")
        text = pat.sub(f"#define {key} {val}", text, count=1)
    return text


def available() -> bool:
    return REF_ROOT is not None and (REF_ROOT / "src" / "cilia" / "cuda_functions.cu").exists()


FCM_SOURCES = ["CUFCM_SOLVER.cu", "CUFCM_FCM.cu", "CUFCM_CORRECTION.cu", "CUFCM_DATA.cu", "CUFCM_CELLLIST.cu",
               "CUFCM_RANDOMPACKER.cu"]
FCM_WRAPPER = HERE / "ref_fcm_wrapper.cu"


def fcm_lib_path() -> Path:
    return OUT / "libref_fcm.so"


def build_fcm(verbose: bool = False, force: bool = False) -> Path | None:
    """The reference's cuFCM (src/cufcm, float build, ROTATION 0 as configured) with ref_fcm_wrapper.cu."""
    if REF_ROOT is None:
        return None
    src_dir = REF_ROOT / "src" / "cufcm"
    if not (src_dir / "CUFCM_SOLVER.cu").exists():
        return None
    OUT.mkdir(exist_ok=True)
    lib = fcm_lib_path()
    srcs = [FCM_WRAPPER] + [src_dir / f for f in FCM_SOURCES]
    newest = max(p.stat().st_mtime for p in srcs)
    if force or not lib.exists() or lib.stat().st_mtime < newest:
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC",
               "-shared", "-I", str(src_dir), *map(str, srcs), "-lcufft", "-lcurand", "-o", str(lib) + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(str(lib) + ".tmp", lib)
    return lib


# The reference's whole prescribed-cilia step (ref_step_harness.cu drives the
# reference's own host code).  Each variant edits switches of config.hpp:
#   step_wgf_f64  the WRITE_GENERALISED_FORCES pre-run, FP64, host RPY back-end
#   step_dyn_f64  the dynamic run, FP64, host RPY back-end (the whole-step CPU oracle)
#   step_dyn_gpu  the dynamic run with the reference's own GPU back-end
#                 (rpy_mobility_solver + Mss_mult), FP32 as the reference ships it
#   step_body_f64 a free spherical body with prescribed cilia (BODY_OR_SURFACE_TYPE 2,
#                 BODY_VELOCITY_TYPE 0), FP64, host unbounded-RPY back-end
#   step_dyn_f64_tight  step_dyn_f64 with GMRES tolerance 1e-10 (near-exact linear solves)
# All others use GMRES tolerance 1e-6 (LINEAR_SYSTEM_TOL) and a Fulford-Blake beat.
STEP_SWITCHES = {"CILIA_TYPE": "3", "BODY_OR_SURFACE_TYPE": "0", "MOBILITY_TYPE": "1", "LINEAR_SYSTEM_TOL": "1e-6",
                 "SHAPE_SEQUENCE": "1", "DYNAMIC_PHASE_EVOLUTION": "true", "DYNAMIC_SHAPE_ROTATION": "true",
                 "INITIAL_CONDITIONS_TYPE": "0", "DISPLAYTIME": "false"}
STEP_VARIANTS = {
    "step_wgf_f64": ({"WRITE_GENERALISED_FORCES": "true", "FIL_USE_DOUBLE_PRECISION": "true"}, False),
    "step_dyn_f64": ({"WRITE_GENERALISED_FORCES": "false", "FIL_USE_DOUBLE_PRECISION": "true"}, False),
    "step_dyn_gpu": ({"WRITE_GENERALISED_FORCES": "false", "FIL_USE_DOUBLE_PRECISION": "false"}, True),
    # a free rigid spherical body carrying prescribed cilia, unbounded RPY (host back-end)
    "step_body_f64": ({"WRITE_GENERALISED_FORCES": "false", "FIL_USE_DOUBLE_PRECISION": "true",
                       "BODY_OR_SURFACE_TYPE": "2", "BODY_VELOCITY_TYPE": "0"}, False),
    "step_dyn_f64_tight": ({"WRITE_GENERALISED_FORCES": "false", "FIL_USE_DOUBLE_PRECISION": "true",
                            "LINEAR_SYSTEM_TOL": "1e-10"}, False),
    # instability-driven elastic cilia on the wall (Broyden's method), driven by ref_elastic_harness.cu
    "elastic_f64": ({"WRITE_GENERALISED_FORCES": "false", "FIL_USE_DOUBLE_PRECISION": "true", "CILIA_TYPE": "0",
                     "CILIA_IC_TYPE": "0"}, False),
}
STEP_HOST_CPP = ["src/cilia/mobility/mobility_solver.cpp", "src/cilia/filament.cpp", "src/cilia/swimmer.cpp",
                 "src/cilia/segment.cpp", "src/cilia/rigid_body.cpp", "src/cilia/broyden_solver.cpp",
                 "src/general/matrix.cpp", "src/general/quaternion.cpp"]
STEP_HOST_CU = ["src/cilia/seeding.cu", "src/general/util.cu", "globals.cu"]
STEP_GPU_CU = ["src/cilia/cuda_functions.cu", "src/cilia/mobility/rpy_mobility_solver.cu"]
STEP_HARNESS = HERE / "ref_step_harness.cu"
ELASTIC_HARNESS = HERE / "ref_elastic_harness.cu"
LAPACK_SHIM = HERE / "lapack_shim.c"
RPY_ORACLE = HERE / "rpy_oracle.c"


def step_path(variant: str) -> Path:
    return OUT / f"ref_{variant}"


def _step_switch_text(extra: dict[str, str]) -> str:
    text = (REF_ROOT / "config.hpp").read_text()
    for key, val in {**STEP_SWITCHES, **extra}.items():
        pat = re.compile(rf"^(\s*)#define {key} \S+", re.M)
        if not pat.search(text):
            raise RuntimeError(f"switch {key} not found in the reference config.hpp")
        text = pat.sub(lambda m: f"{m.group(1)}#define {key} {val}", text, count=1)
    return text


def build_step(verbose: bool = False, force: bool = False) -> list[Path]:
    """Builds the step-harness variants into oracle/_ref/ (objects under oracle/_ref/obj_<variant>/)."""
    if not available():
        return []
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    inc = ["-I", str(REF_ROOT), "-I", str(REF_ROOT / "src" / "cilia"), "-I", str(REF_ROOT / "src" / "cilia" / "mobility"),
           "-I", str(REF_ROOT / "src" / "general")]
    arch = ["-gencode", "arch=compute_100a,code=sm_100a"]
    built = []
    for name, (extra, gpu) in STEP_VARIANTS.items():
        odir = OUT / f"obj_{name}"
        odir.mkdir(parents=True, exist_ok=True)
        cfg = odir / "config_variant.hpp"
        text = _step_switch_text(extra)
        if force or not cfg.exists() or cfg.read_text() != text:
            cfg.write_text(text)
        jobs = []  # (source, object, command prefix)
        for rel in STEP_HOST_CPP:
            src = REF_ROOT / rel
            jobs.append((src, odir / (src.stem + ".o"),
                         ["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-include", str(cfg), *inc,
                          "-I", "/usr/local/cuda/include", "-c", str(src)]))
        for rel in STEP_HOST_CU + (STEP_GPU_CU if gpu else []):
            src = REF_ROOT / rel
            jobs.append((src, odir / (src.stem + ".o"),
                         [nvcc, *arch, "-std=c++17", "-O2", "-w", "-x", "cu", "-include", str(cfg), *inc,
                          "-c", str(src)]))
        harness = ELASTIC_HARNESS if name.startswith("elastic") else STEP_HARNESS
        jobs.append((harness, odir / (harness.stem + ".o"),
                     [nvcc, *arch, "-std=c++17", "-O2", "-w", "-include", str(cfg), *inc,
                      *(["-DREF_HARNESS_GPU"] if gpu else []), "-c", str(harness)]))
        jobs.append((LAPACK_SHIM, odir / "lapack_shim.o", ["gcc", "-O2", "-std=c11", "-c", str(LAPACK_SHIM)]))
        if not gpu:
            jobs.append((RPY_ORACLE, odir / "rpy_oracle_f64.o",
                         ["gcc", "-O2", "-fopenmp", "-std=c11", "-c", str(RPY_ORACLE)]))
        objs = []
        for src, obj, cmd in jobs:
            objs.append(obj)
            if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, cfg.stat().st_mtime):
                if verbose:
                    print(" ".join(cmd + ["-o", str(obj)]), file=sys.stderr)
                subprocess.run(cmd + ["-o", str(obj)], check=True)
        exe = step_path(name)
        if force or not exe.exists() or exe.stat().st_mtime < max(o.stat().st_mtime for o in objs):
            cmd = [nvcc, *arch, "-o", str(exe) + ".tmp", *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            os.replace(str(exe) + ".tmp", exe)
        built.append(exe)
    return built


FLOW_WRAPPER = HERE / "ref_flow_wrapper.cu"


def flow_lib_path() -> Path:
    return OUT / "libref_flow.so"


def build_flow(verbose: bool = False, force: bool = False) -> Path | None:
    """The reference's flow_velocities kernel (src/flow_field/flow_field_evaluator.cu) in FP64, with the
    reference's matrix/quaternion sources it links against and the BLAS/LAPACK shim."""
    if not available():
        return None
    src = REF_ROOT / "src" / "flow_field" / "flow_field_evaluator.cu"
    if not src.exists():
        return None
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    odir = OUT / "obj_flow"
    odir.mkdir(parents=True, exist_ok=True)
    cfg = odir / "config_variant.hpp"
    text = _step_switch_text({"FIL_USE_DOUBLE_PRECISION": "true", "WRITE_GENERALISED_FORCES": "false"})
    if force or not cfg.exists() or cfg.read_text() != text:
        cfg.write_text(text)
    inc = ["-I", str(REF_ROOT), "-I", str(REF_ROOT / "src" / "general"), "-I", str(REF_ROOT / "src" / "flow_field")]
    jobs = [(REF_ROOT / "src" / "general" / "matrix.cpp", odir / "matrix.o",
             ["g++", "-std=c++17", "-O2", "-fPIC", "-w", "-include", str(cfg), *inc, "-c"]),
            (REF_ROOT / "src" / "general" / "quaternion.cpp", odir / "quaternion.o",
             ["g++", "-std=c++17", "-O2", "-fPIC", "-w", "-include", str(cfg), *inc, "-c"]),
            (LAPACK_SHIM, odir / "lapack_shim.o", ["gcc", "-O2", "-fPIC", "-std=c11", "-c"]),
            (FLOW_WRAPPER, odir / "ref_flow_wrapper.o",
             [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC",
              "-include", str(cfg), *inc, "-c"])]
    objs = []
    for s_, o_, cmd in jobs:
        objs.append(o_)
        newest = max(s_.stat().st_mtime, cfg.stat().st_mtime, src.stat().st_mtime)
        if force or not o_.exists() or o_.stat().st_mtime < newest:
            if verbose:
                print(" ".join(cmd + [str(s_), "-o", str(o_)]), file=sys.stderr)
            subprocess.run(cmd + [str(s_), "-o", str(o_)], check=True)
    lib = flow_lib_path()
    if force or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(lib) + ".tmp",
               *map(str, objs)]
        subprocess.run(cmd, check=True)
        os.replace(str(lib) + ".tmp", lib)
    return lib


def build(verbose: bool = False, force: bool = False) -> list[Path]:
    """Builds every variant; a no-op returning [] when the reference tree is absent."""
    if not available():
        return []
    OUT.mkdir(exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    built = []
    for name, sw in VARIANTS.items():
        cfg = OUT / f"config_{name}.hpp"
        lib = lib_path(name)
        text = _config_text(sw)
        if force or not cfg.exists() or cfg.read_text() != text:
            cfg.write_text(text)
        src_cu = REF_ROOT / "src" / "cilia" / "cuda_functions.cu"
        newest = max(cfg.stat().st_mtime, WRAPPER.stat().st_mtime, src_cu.stat().st_mtime)
        if force or not lib.exists() or lib.stat().st_mtime < newest:
            cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-w",
                   "-Xcompiler", "-fPIC", "-shared", "-include", str(cfg),
                   "-I", str(REF_ROOT / "src" / "cilia"), "-I", str(REF_ROOT),
                   str(WRAPPER), "-o", str(lib) + ".tmp"]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            os.replace(str(lib) + ".tmp", lib)
        built.append(lib)
    fcm = build_fcm(verbose, force)
    if fcm is not None:
        built.append(fcm)
    built.extend(build_step(verbose, force))
    flow = build_flow(verbose, force)
    if flow is not None:
        built.append(flow)
    return built


if __name__ == "__main__":
    # python oracle/ref_build.py REFERENCE_ROOT [--force]
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if args:
        set_reference_root(args[0])
    for p in build(verbose=True, force="--force" in sys.argv):
        print(p)
