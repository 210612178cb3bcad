"""Builds libemsesg.so (the sm_100a kernels and the C ABI) in-tree with nvcc.

    python -m ctca_b200.build          # or: from ctca_b200.build import build; build()

dropin.cu is compiled with --fmad=false: the plain FP64 drop-in keeps the
reference's IEEE operation sequence without fused multiply-adds.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libemsesg.so"
BUILD_DIR = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          f"-I{INCLUDE}"]
SOURCES = {
    "context.cu": [],
    "dropin.cu": ["--fmad=false"],
    "sort.cu": [],
    "fx.cu": [],
    "noalloc.cu": [],
    "esfield.cu": [],
}
LIBS = ["-lcufft"]  # the electrostatic field step's FFTs


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libemsesg")
    return path


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [INCLUDE / "emses_gpu.h", Path(__file__)]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None) -> Path:
    BUILD_DIR.mkdir(exist_ok=True)
    objs = []
    for name, flags in SOURCES.items():
        src = CSRC / name
        obj = BUILD_DIR / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra or []), "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), *LIBS]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
