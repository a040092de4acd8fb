"""Build the native library ``voxviz_b200/libvoxviz_b200.so`` in tree.

CUDA sources are compiled for sm_100a only, with IEEE division and square
root and without FMA contraction (the kernels' integer decisions must match
the host arithmetic bit for bit).  Host C++ is compiled with
``-ffp-contract=off`` for the same reason (the terrain heights are
reproduced exactly by the checks).  Objects go to ``voxviz_b200/_build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libvoxviz_b200.so"
INCLUDE = PKG.parent / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
HOST_CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"

CU_SOURCES = ["kernels.cu", "ctx.cu", "noalloc.cu", "production.cu", "adjoint.cu", "batch.cu", "builder.cu",
              "compact.cu"]
CPP_SOURCES = ["terrain.cpp", "octree.cpp", "gradients.cpp", "gvfile.cpp", "renderer.cpp", "scene.cpp", "capi.cpp"]
HEADERS = ["kernels.cuh", "cellmask.cuh", "select.cuh", "compact.h", "dxt.h", "ctx.h", "terrain.h", "octree.h", "gvfile.h", "scene.h", "handles.h", "renderer.h", "production.h", "raycast_common.cuh",
           "lod_bound.h", "gradients.h", "fixed_div.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-ccbin", HOST_CXX,
]
CXX_FLAGS = [
    "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
    "-march=x86-64-v2", "-Wall", "-Wextra", "-Wno-unused-parameter",
    f"-I{CUDA_HOME / 'include'}",
]


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every source that changed and link the shared library."""
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "voxviz_b200.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC, *NVCC_FLAGS, *extra, "-c", str(s), "-o", str(o)])
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            jobs.append([HOST_CXX, *CXX_FLAGS, "-c", str(s), "-o", str(o)])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for cmd in jobs:
                if verbose:
                    print(" ".join(cmd))
            list(ex.map(_run, jobs))
    if jobs or not LIB.exists() or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, "-shared", "-ccbin", HOST_CXX, "-o", str(tmp), *map(str, objs),
              "-Xcompiler", "-fopenmp", "-lgomp"])
        shutil.move(str(tmp), str(LIB))
    return LIB


if __name__ == "__main__":
    info = "--ptxas" in sys.argv
    print(build(verbose="-v" in sys.argv, ptxas_info=info))
