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
REF_ROOT = Path(os.environ.get("CUFIL_REFERENCE_ROOT", "/root/reference"))
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
    return (REF_ROOT / "src" / "cilia" / "cuda_functions.cu").exists()


FCM_SOURCES = ["CUFCM_SOLVER.cu", "CUFCM_FCM.cu", "CUFCM_CORRECTION.cu", "CUFCM_DATA.cu", "CUFCM_CELLLIST.cu",
               "CUFCM_RANDOMPACKER.cu"]
FCM_WRAPPER = HERE / "ref_fcm_wrapper.cu"


def fcm_lib_path() -> Path:
    return OUT / "libref_fcm.so"


def build_fcm(verbose: bool = False, force: bool = False) -> Path | None:
    """The reference's cuFCM (src/cufcm, float build, ROTATION 0 as configured) with ref_fcm_wrapper.cu."""
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
    return built


if __name__ == "__main__":
    for p in build(verbose=True, force="--force" in sys.argv):
        print(p)
