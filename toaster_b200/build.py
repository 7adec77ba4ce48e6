"""Builds the in-tree CUDA library (sm_100a) with nvcc.

    python -m toaster_b200.build

produces ``toaster_b200/lib/libtoaster_cuda.so`` (loaded through ctypes) and
``toaster_b200/lib/libtoaster_cuda.a`` (for a native host such as the Rust crate
``toaster-cuda``). Host C++ is compiled with -ffp-contract=off: the hierarchy bounds must round
exactly like the reference's f32 arithmetic.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
SOURCES = ["api.cu", "kernels.cu", "guide.cu", "umma_selftest.cu", "display.cu", "refit.cu", "bvh_device.cu",
           "probe.cu",
           "bvh_build.cpp", "scene_loader.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def common_flags() -> list:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   f"-I{PKG.parent / 'include'}"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the shared and static libraries if any source changed; returns the .so path."""
    LIB.mkdir(parents=True, exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
    deps.append(PKG.parent / "include" / "toaster_cuda.h")
    so = LIB / "libtoaster_cuda.so"
    if not force and not _stale(so, deps):
        return so
    objdir = LIB / "obj"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc()] + common_flags() + ["-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = so.with_suffix(".so.tmp")
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lnvjpeg", "-lz"], check=True)
    os.replace(tmp, so)
    static = LIB / "libtoaster_cuda.a"
    if static.exists():
        static.unlink()
    subprocess.run([nvcc()] + ARCH + ["-lib", "-o", str(static)] + objs, check=True)
    return so


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB / "libtoaster_cuda.so")
