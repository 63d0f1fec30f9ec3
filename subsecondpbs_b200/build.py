"""Builds libsubsecondpbs_b200.so in-tree with nvcc for sm_100a.

Usage: python -m subsecondpbs_b200.build [--force]

Host C++ is compiled without floating-point contraction so the host planner's
float arithmetic is evaluated exactly as written (the beam-grid integer decisions
depend on it). Device code is compiled for sm_100a only.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libsubsecondpbs_b200.so"
BUILD_DIR = PKG / "_build"

CU_SOURCES = ["trace.cu", "conv.cu", "idd.cu", "superpose.cu", "transfer.cu", "context.cu", "peak.cu", "noalloc.cu", "adjoint.cu", "operator.cu", "bio.cu"]
CXX_SOURCES = ["plan.cpp", "capi.cpp", "final_dose.cpp", "server.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build subsecondpbs_b200")
    return exe


def _sources() -> list[Path]:
    return [CSRC / s for s in CU_SOURCES + CXX_SOURCES]


def _deps() -> list[Path]:
    return _sources() + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD_DIR.mkdir(exist_ok=True)
    objs = []
    cc = nvcc()
    for src in _sources():
        obj = BUILD_DIR / (src.name + ".o")
        cmd = [cc, *ARCH, *COMMON, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cuda_inc = str(Path(cc).resolve().parent.parent / "include")
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-I", cuda_inc,
                   "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    link = [cc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
