"""Build the CPU oracle (test infrastructure) as oracle/liboracle.so.

g++ -O2 -ffp-contract=off: no fused multiply-add, so every expression
rounds as its sequential left-to-right evaluation, like the GPU library
built with --fmad=false.  -fopenmp: the solver runs one emulated rank
(preconditioner block) per thread and its cell loops in parallel, with
results identical to one thread (OMP_NUM_THREADS sets the count).
"""
from __future__ import annotations

import os
import pathlib
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRC = HERE / "oracle.cpp"


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [SRC, HERE / "oracle.h", HERE.parent / "include" / "cadmas_gpu.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False) -> pathlib.Path:
    if not force and not needs_build():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-Wall", "-o", str(tmp), str(SRC)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
