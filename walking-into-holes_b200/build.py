"""Build libtwos.so and the wih_twos / wih_adjoint executables in-tree.

    python walking-into-holes_b200/build.py [--force]

Everything is compiled by nvcc for sm_100a only (-gencode
arch=compute_100a,code=sm_100a) into walking-into-holes_b200/_build/.  The
CUDA runtime is linked statically so the library does not depend on the
runtime version another library in the process (e.g. torch) brings.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "_build"
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I", str(CSRC)]
CUDA_FLAGS = ARCH + ["-lineinfo", "-fmad=false", "--expt-relaxed-constexpr"]

LIB_SOURCES = ["kernels.cu", "design.cu", "noalloc.cu", "twos_abi.cpp", "geometry.cpp"]
# Executables: name -> (source, extra defines).  The study variants mirror the
# reference's macro builds of study.cpp (analytic_query.cpp, compliance_query.cpp).
CLI = {
    "wih_twos": ("cli_twos.cpp", []),
    "wih_adjoint": ("cli_adjoint.cpp", []),
    "wih_study": ("cli_study.cpp", []),
    "wih_analytic_query": ("cli_study.cpp", ["-DTWOS_STUDY_ANALYTIC=1"]),
    "wih_compliance_query": ("cli_study.cpp", ["-DTWOS_STUDY_ANALYTIC=1", "-DTWOS_STUDY_AFFINE=1"]),
    "wih_analytic_integral_audit": ("cli_audit.cpp", []),
}
HEADERS = ["twos_internal.h", "twos_session.h", "cli_common.h", "diffwos.cuh", "ball_green.cuh", "validate.cuh", "rqmc.cuh",
           "wavefront.cuh"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def host_compiler() -> list[str]:
    # nvcc's host compiler: the system g++ (the CXX variable of some images
    # points at a compiler without the libraries the build needs).
    gxx = shutil.which("g++", path="/usr/bin") or shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    OUT.mkdir(parents=True, exist_ok=True)
    headers = [CSRC / h for h in HEADERS if (CSRC / h).exists()] + [INCLUDE / "twos.h"]
    objs = []
    for src in LIB_SOURCES:
        s = CSRC / src
        o = OUT / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            flags = CUDA_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) if s.suffix == ".cu" else []
            run([nvcc()] + host_compiler() + COMMON + flags + ["-c", str(s), "-o", str(o)])
    lib = OUT / "libtwos.so"
    if force or _stale(lib, objs):
        run([nvcc()] + host_compiler() + ARCH + ["-shared", "-cudart", "static", "-o", str(lib)]
            + [str(o) for o in objs] + ["-lpthread"])
    for exe, (src, defines) in CLI.items():
        s = CSRC / src
        target = OUT / exe
        if force or _stale(target, [s, lib] + headers):
            run([nvcc()] + host_compiler() + COMMON + defines + ["-o", str(target), str(s), "-L", str(OUT),
                 "-ltwos", "-Xlinker", "-rpath,$ORIGIN"])
    return lib


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args()
    build(force=a.force, verbose_ptxas=a.ptxas)


if __name__ == "__main__":
    sys.exit(main())
