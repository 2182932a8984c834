"""Builds the twins-b200 native code in-tree for sm_100a.

    python -m twins_b200.build            # the libraries and the twins / twins128 front-ends
    python -m twins_b200.build --force

Outputs (git-ignored, they travel with the repository to the GPU machine):
    twins_b200/lib/libtwinsb200.so        the C ABI of include/twinsb200.h (9-run event chains)
    twins_b200/lib/twins                  the reference's command line over it
    twins_b200/lib/libtwinsb200_runs25.so the same with 25-run chains (128-byte frames), as the
    twins_b200/lib/twins128               reference's twins128 build (-DTWINS_CHAIN_RUNS=25)
    twins_b200/lib/libtwinsb200_trace.so  the same recording every enqueue (the reference's
    twins_b200/lib/twins-trace            --qtrace); twins runs twins-trace when given --qtrace
    twins_b200/lib/twins-rdma             the reference's RDMA command line over libtwinsb200.so
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
SO25 = LIB / "libtwinsb200_runs25.so"
CLI25 = LIB / "twins128"
SO_TRACE = LIB / "libtwinsb200_trace.so"
CLI_TRACE = LIB / "twins-trace"
CLI_RDMA = LIB / "twins-rdma"
# (library, front-end, extra flags): 9-run chains, 25-run chains, 9-run chains with the enqueue trace
VARIANTS = [(SO, CLI, []), (SO25, CLI25, ["-DTB_CHAIN_RUNS=25"]), (SO_TRACE, CLI_TRACE, ["-DTB_QTRACE"])]
# (on request: the RDMA slot kernel's timers of the slots' longest NIC and switch, TR_PROFILE)
SO_PROF = LIB / "libtwinsb200_prof.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# exactness: no floating-point contraction (fma() is written where ns-3 fuses), IEEE division
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"] + ARCH
SOURCES = ["tb_kernel.cu", "tb_capi.cu", "tr_kernel.cu", "tr_capi.cu"]


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


def build_profile() -> Path:
    """The profiling build (TR_PROFILE counters in the RDMA slot kernel), for measurements only."""
    LIB.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in SOURCES:
        obj = LIB / (Path(src).stem + "_prof.o")
        subprocess.run([nvcc, *NVFLAGS, "-DTR_PROFILE", "-c", str(CSRC / src), "-o", str(obj)], check=True)
        objs.append(str(obj))
    subprocess.run([nvcc, *ARCH, "-shared", "-o", str(SO_PROF), *objs, "-lcudart"], check=True)
    for o in objs:
        Path(o).unlink(missing_ok=True)
    return SO_PROF


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    deps = [d for d in list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))] + \
        [ROOT / "include" / "twinsb200.h", Path(__file__)]
    nvcc = _nvcc()
    # every stale library's objects compile at once (each is one nvcc process), then link
    jobs, links = [], []
    for so, cli, extra in VARIANTS:
        if force or _stale(so, deps):
            objs = []
            for src in SOURCES:
                obj = LIB / (Path(src).stem + so.stem + ".o")
                cmd = [nvcc, *NVFLAGS, *extra, "-c", str(CSRC / src), "-o", str(obj)]
                if verbose:
                    print(" ".join(cmd))
                jobs.append(subprocess.Popen(cmd))
                objs.append(str(obj))
            links.append((so, objs))
    failed = [j.args for j in jobs if j.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    for so, objs in links:
        subprocess.run([nvcc, *ARCH, "-shared", "-o", str(so), *objs, "-lcudart"], check=True)
        for o in objs:
            Path(o).unlink(missing_ok=True)
    for so, cli, extra in VARIANTS:
        if force or _stale(cli, deps + [so]):
            cmd = ["g++", "-std=c++17", "-O2", "-o", str(cli), str(CSRC / "twins_cli.cpp"),
                   f"-L{LIB}", f"-l{so.stem[3:]}", f"-Wl,-rpath,$ORIGIN"]
            subprocess.run(cmd, check=True)
    if force or _stale(CLI_RDMA, deps + [SO]):
        subprocess.run(["g++", "-std=c++17", "-O2", "-o", str(CLI_RDMA), str(CSRC / "twins_rdma_cli.cpp"), f"-L{LIB}", "-ltwinsb200",
                        "-Wl,-rpath,$ORIGIN"], check=True)
    return SO


if __name__ == "__main__":
    if "--profile" in sys.argv:
        print(build_profile())
        sys.exit(0)
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(SO)
