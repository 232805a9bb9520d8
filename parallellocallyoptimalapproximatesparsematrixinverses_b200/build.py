"""Builds libspai_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ with a C ABI (no torch, no Python in the
signatures).  FMA contraction is disabled (--fmad=false) so the FP64 path
rounds every product and sum separately, as the reference's x86-64 build does;
the kernels that want FMA in FP32 call it explicitly.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR / "csrc"
LIB_PATH = PACKAGE_DIR / "libspai_b200.so"
BUILD_DIR = PACKAGE_DIR / "_build"

SOURCES = ["ops.cu", "spgemm.cu", "update.cu", "solver.cu", "mr_fused.cu", "pcg.cu", "c_api.cu", "profile.cu", "noalloc.cu",
           "adjoint.cu", "mtx.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "-Xptxas", "-O3",
]


def nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda_home) / "bin" / "nvcc"
    return str(candidate) if candidate.exists() else "nvcc"


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    newest_header = max((p.stat().st_mtime for p in CSRC.glob("*.cuh")), default=0.0)
    include_headers = max((p.stat().st_mtime for p in (PACKAGE_DIR.parent / "include").glob("*.h")), default=0.0)
    return obj.stat().st_mtime < max(src.stat().st_mtime, newest_header, include_headers, Path(__file__).stat().st_mtime)


def build(verbose: bool = False, jobs: int = 5) -> Path:
    """Compile every .cu into an object and link the shared library."""
    BUILD_DIR.mkdir(exist_ok=True)
    objects = []
    procs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD_DIR / (name + ".o")
        objects.append(obj)
        if _stale(obj, src):
            cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((name, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            if len(procs) >= jobs:
                _wait(procs)
                procs = []
    _wait(procs)
    needs_link = not LIB_PATH.exists() or any(o.stat().st_mtime > LIB_PATH.stat().st_mtime for o in objects)
    if needs_link:
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB_PATH),
               *map(str, objects), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB_PATH


def _wait(procs) -> None:
    failed = []
    for name, proc in procs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            failed.append((name, out.decode(errors="replace")))
        elif out:
            text = out.decode(errors="replace").strip()
            if text:
                print(text)
    if failed:
        for name, text in failed:
            print(f"--- nvcc failed on {name} ---\n{text}", file=sys.stderr)
        raise RuntimeError("nvcc failed: " + ", ".join(n for n, _ in failed))


if __name__ == "__main__":
    print(build(verbose=True))
