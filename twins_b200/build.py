"""Builds the twins-b200 native code in-tree for sm_100a.

    python -m twins_b200.build            # libtwinsb200.so and the twins front-end
    python -m twins_b200.build --force

Outputs (git-ignored, they travel with the repository to the GPU machine):
    twins_b200/lib/libtwinsb200.so    the C ABI of include/twinsb200.h
    twins_b200/lib/twins              the reference's command line over it
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
SO = LIB / "libtwinsb200.so"
CLI = LIB / "twins"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# exactness: no floating-point contraction (fma() is written where ns-3 fuses), IEEE division
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"] + ARCH
SOURCES = ["tb_kernel.cu", "tb_capi.cu"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or Path(c).exists()):
            return c
    return "nvcc"


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        [ROOT / "include" / "twinsb200.h", Path(__file__)]
    nvcc = _nvcc()
    if force or _stale(SO, deps):
        objs = []
        for src in SOURCES:
            obj = LIB / (Path(src).stem + ".o")
            cmd = [nvcc, *NVFLAGS, "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(str(obj))
        cmd = [nvcc, *ARCH, "-shared", "-o", str(SO), *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
        for o in objs:
            Path(o).unlink(missing_ok=True)
    if force or _stale(CLI, deps + [SO]):
        cmd = ["g++", "-std=c++17", "-O2", "-o", str(CLI), str(CSRC / "twins_cli.cpp"),
               f"-L{LIB}", "-ltwinsb200", f"-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(SO)
