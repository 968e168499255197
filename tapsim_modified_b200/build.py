"""Builds libtapsim_b200.so in-tree: sm_100a device code (nvcc) plus the C++
host library (mesh generation, Delaunay, Voronoi tables, file formats).

    python -m tapsim_modified_b200.build          # incremental
    python -m tapsim_modified_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libtapsim_b200.so"
PROGRAM = PKG / "tapsim_b200"
HOST_PROGRAM = "host/tapsim_b200.cpp"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["relax.cu", "cg.cu", "amg.cu", "surface.cu", "flight.cu", "mpnn.cu", "learn.cu", "handle.cu"]
CPP_SOURCES = ["host/tipgen.cpp", "host/samplegen.cpp", "host/delaunay.cpp", "host/voronoi.cpp", "host/formats.cpp", "host/mesh_api.cpp",
               "host/amg.cpp", "host/amg_api.cpp"]
HEADERS = ["device_common.cuh", "kernels.cuh", "host/tipgen.h", "host/samplegen.h", "host/delaunay.h", "host/voronoi.h",
           "host/formats.h", "host/predicates.h", "host/amg.h"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    deps = [CSRC / h for h in HEADERS] + [ROOT / "include" / "tapsim_gpu.h"]
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (Path(src).stem + ".cu.o")
        objs.append(o)
        if force or _stale(o, s, deps):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c", str(s), "-o", str(o)]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            _run(cmd)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (Path(src).stem + ".o")
        objs.append(o)
        if force or _stale(o, s, deps):
            _run([CXX, "-O2", "-std=c++17", "-fPIC", "-pthread", "-c", str(s), "-o", str(o)])
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
              "-Xcompiler", "-pthread", "-lpthread"])
    # the C++ host program over the C ABI (evaporation / resumption
    # commands), linked against the in-tree library
    src = CSRC / HOST_PROGRAM
    if force or _stale(PROGRAM, src, [ROOT / "include" / "tapsim_gpu.h", LIB]):
        _run([CXX, "-O2", "-std=c++17", "-o", str(PROGRAM), str(src), f"-L{PKG}", "-ltapsim_b200",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
