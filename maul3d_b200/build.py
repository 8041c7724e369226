"""Build recipe for libmaul3d_b200.so (in-tree, no JIT cache).

Device code is compiled for sm_100a only, with the determinism flags the
bit-exact contract needs: no fused multiply-add contraction
(-fmad=false), IEEE-rounded division and square root (-prec-div=true
-prec-sqrt=true) and denormals preserved (-ftz=false).  Host code is
compiled with -ffp-contract=off, like the reference engine's own build.

Run `python maul3d_b200/build.py` (or __graft_entry__.build()).  The
CUDA runtime is linked statically so the library has no runtime search
path requirements beyond the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libmaul3d_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DET_DEVICE = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
DET_HOST = ["-ffp-contract=off", "-fno-fast-math", "-fno-unsafe-math-optimizations"]

CU_SOURCES = ["step.cu", "hash.cu", "upload.cu"]
CPP_SOURCES = ["world.cpp", "device.cpp", "capi.cpp", "hostmem.cpp", "snapshot.cpp", "serve.cpp",
               "events.cpp", "quickhull.cpp"]
C_SOURCES = ["scenes.c"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile every source that changed and link the shared library."""
    if not Path(NVCC).exists() and shutil.which("nvcc") is None:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    objs: list[Path] = []
    inc = [f"-I{INCLUDE}", f"-I{CSRC}"]
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", *DET_DEVICE,
                   "-Xcompiler", "-fPIC," + ",".join(DET_HOST), *inc, "-c", str(s), "-o", str(o)]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd, verbose)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", *DET_HOST, *inc,
                  f"-I{CUDA_HOME / 'include'}", "-c", str(s), "-o", str(o)], verbose)
    for src in C_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run(["gcc", "-O2", "-std=c17", "-fPIC", "-fvisibility=hidden", *DET_HOST, *inc,
                  "-c", str(s), "-o", str(o)], verbose)
    if force or _stale(LIB, objs):
        _run(["g++", "-shared", "-o", str(LIB), *map(str, objs),
              f"-L{CUDA_HOME / 'lib64'}", "-lcudart_static", "-ldl", "-lrt", "-lpthread",
              "-Wl,--exclude-libs,ALL"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
