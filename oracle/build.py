"""Build recipe for the oracle's C restatement (test infrastructure only).

Compiles ``rpy_oracle.c`` twice (FP64 and FP32 arithmetic) with OpenMP into
``oracle/_build/liboracle_rpy.so``.  The tests, ``__graft_entry__.smoke`` and
the CPU-baseline leg of ``bench.py`` load it as the checker; the product never
does.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "liboracle_rpy.so"
SRC = HERE / "rpy_oracle.c"
CFLAGS = ["-O2", "-fPIC", "-fopenmp", "-Wall", "-Wextra", "-std=c11"]


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    o64 = BUILD / "rpy_oracle_f64.o"
    o32 = BUILD / "rpy_oracle_f32.o"
    cmds = [
        ["gcc", *CFLAGS, "-c", str(SRC), "-o", str(o64)],
        ["gcc", *CFLAGS, "-DORACLE_REAL=float", "-DORACLE_SUFFIX=f32", "-c", str(SRC), "-o", str(o32)],
        ["gcc", "-shared", "-fopenmp", "-o", str(LIB) + ".tmp", str(o64), str(o32), "-lm"],
    ]
    for c in cmds:
        if verbose:
            print(" ".join(c), file=sys.stderr)
        subprocess.run(c, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
