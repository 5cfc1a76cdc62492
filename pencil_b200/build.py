"""Build libpencil_gpu.so (sm_100a) in-tree.

The library is the CUDA kernels plus the C-ABI of include/pencil_gpu.h. Device
code is compiled with --fmad=false and IEEE division/square root so that every
float operation rounds as Pencil's x86-64 build does; host code with
-ffp-contract=off for the same reason.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libpencil_gpu.so"
INCLUDE = HERE.parent / "include"

CU_SOURCES = ["api.cu", "megakernel.cu", "wavefront.cu", "queries.cu", "adjoint.cu",
              "tonemap.cu", "bvh_device.cu"]
CXX_SOURCES = ["bvh_build.cpp", "bvh_wide.cpp", "host_pool.cpp"]
HEADERS = ["device_common.cuh", "path.cuh", "scene_layout.h", "host_internal.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", str(INCLUDE),
]
CUDA_INCLUDE = "/usr/local/cuda/include"
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", str(INCLUDE), "-I", CUDA_INCLUDE]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpencil_gpu.so")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + proc.stdout + proc.stderr)


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None) -> Path:
    """Compile the library if any source is newer than it; returns its path."""
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "pencil_gpu.h"]
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([nvcc] + NVCC_FLAGS + (extra or []) + ["-c", str(src), "-o", str(obj)])
    for s in CXX_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for cmd, fut in [(j, ex.submit(_run, j)) for j in jobs]:
                if verbose:
                    print(" ".join(cmd), file=sys.stderr)
                fut.result()
    if force or jobs or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lcudart_static"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
