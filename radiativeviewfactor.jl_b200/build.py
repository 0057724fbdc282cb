"""Build librvf_b200.so in-tree (lib/) with nvcc for sm_100a.

Every translation unit is compiled with --fmad=false / -ffp-contract=off:
the device reproduces the reference's Float64 evaluation order exactly and
requests fused multiply-adds explicitly where a tolerance allows them.
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
LIBDIR = HERE / "lib"
OBJDIR = HERE / "_build"
LIB = LIBDIR / "librvf_b200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I", str(CSRC), "-I", str(INCLUDE),
] + os.environ.get("RVF_NVCC_DEFINES", "").split()  # tuning macros, e.g. -DRVF_PAIR_MIN_BLOCKS=3


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile (if stale) and return the path of lib/librvf_b200.so."""
    nvcc = _nvcc()
    LIBDIR.mkdir(exist_ok=True)
    OBJDIR.mkdir(exist_ok=True)
    hdr_mtime = max((p.stat().st_mtime for p in _headers()), default=0.0)
    objs, todo = [], []
    for src in _sources():
        obj = OBJDIR / (src.name + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime)
        if stale:
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [nvcc, *NVCC_FLAGS, "-x", "cu", "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stdout.write(f"compiled {src.name}\n")
        return r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(todo))) as ex:
            list(ex.map(compile_one, todo))
    newest = max(o.stat().st_mtime for o in objs)
    if force or todo or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stdout.write(f"linked {LIB}\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
