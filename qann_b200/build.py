"""Builds the qann_b200 native library in-tree: qann_b200/libqann_gpu.so.

Every CUDA source is compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) with ``-fmad=false`` (the search path's
float arithmetic must round exactly as the reference's CPU build does; the
kernels use explicit fused-multiply-add intrinsics where the reference fuses).
Objects go to ``_build/``; only changed sources are recompiled.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
OUT = PKG / "libqann_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++20", "-O3", "-fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}"]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-Wall", "-ffp-contract=off"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and pathlib.Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "qann_gpu.h"]


def _stale(src: pathlib.Path, obj: pathlib.Path, newest_header: float) -> bool:
    return not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)


def _compile(src: pathlib.Path, obj: pathlib.Path, verbose: bool):
    if src.suffix == ".cu":
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [os.environ.get("CXX", "g++"), *CXX_FLAGS, f"-I{ROOT / 'include'}",
               "-I/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    newest = max(h.stat().st_mtime for h in _headers())
    objs, todo = [], []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if _stale(s, o, newest):
            todo.append((s, o))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for msg in ex.map(lambda so: _compile(*so, verbose), todo):
                if verbose and msg:
                    print(msg)
    if todo or not OUT.exists() or OUT.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = OUT.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking failed:\n{r.stdout}\n{r.stderr}")
        tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
