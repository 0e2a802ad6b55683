"""Build recipe for libcufil.so (sm_100a only).

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a``/``sm_100a`` into
``cufcm_fil_b200/libcufil.so`` next to this file, so the library travels with
the source tree.  Objects are cached under ``cufcm_fil_b200/_build`` and only
recompiled when a source or header is newer than its object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcufil.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fvisibility=hidden"]
LINK_LIBS = ["-lcufft", "-lcuda"]
# The FP32 pair kernels: flush denormals and use the hardware reciprocal / square-root
# approximations (positions and forces are O(1e-3..1e3); the sums are checked against FP64).
PER_FILE_FLAGS = {"rpy_kernels.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcufil.so")
    return cand


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile (incrementally) and link libcufil.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    if not sources:
        raise RuntimeError(f"no CUDA sources under {CSRC}")
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if not stale:
            continue
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *PER_FILE_FLAGS.get(src.name, []), "-I", str(INCLUDE), "-c", str(src),
               "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    lib_stale = force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs)
    if lib_stale:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), *LINK_LIBS]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
