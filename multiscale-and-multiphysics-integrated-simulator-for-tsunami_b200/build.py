"""Build libcadmas_gpu.so in place (sm_100a, FP64 with --fmad=false).

The library is compiled from csrc/*.cu by nvcc directly; the shared object
lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libcadmas_gpu.so"
SOURCES = ["api.cu", "k_momentum.cu", "k_poisson.cu", "k_vof.cu", "k_bc.cu", "k_drop.cu", "k_slope.cu", "k_keps.cu", "k_unet.cu", "unet.cu", "warmstart.cu", "noalloc.cu", "wavetheory.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "--fmad=false", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcadmas_gpu.so")
    return cand


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
    deps.append(HERE.parent / "include" / "cadmas_gpu.h")
    return any(d.stat().st_mtime > t for d in deps if d.exists())


OBJ = HERE / "_build"


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile each source to an object file in parallel (no device code
    crosses files), then link the shared object."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    OBJ.mkdir(exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "-shared"]
    cmds = [[nvcc(), *ARCH, *compile_flags, "-c", "-o", str(OBJ / (s[:-3] + ".o")), str(CSRC / s)]
            for s in SOURCES]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for c, r in zip(cmds, results):
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(c)}\n{r.stdout}{r.stderr}")
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *[str(OBJ / (s[:-3] + ".o")) for s in SOURCES]]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
