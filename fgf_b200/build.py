"""Build libfgfcuda.so in-tree (sm_100a) and the oracle's C library.

Each translation unit is compiled to an object in parallel (the kernels are
self-contained per file, so no relocatable device code is needed), then the
objects are linked into one shared library.

Usage: python -m fgf_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libfgfcuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["kernels.cu", "batch.cu", "gf2mma.cu", "wide.cu", "api.cpp", "tables.cpp", "serve.cpp", "decode.cpp",
           "tune.cpp"]
FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _compile(src: Path, headers: list[Path], force: bool, verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    if force or _stale(obj, [src, *headers]):
        cmd = [NVCC, *FLAGS, "-c", "-o", str(obj), str(src)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return obj


def build_lib(force: bool = False, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "fgf_cuda.h"]
    if not force and not _stale(LIB, srcs + headers):
        return LIB
    OBJ.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, headers, force, verbose), srcs))
    cmd = [NVCC, *ARCH, "--shared", "-cudart", "static", "-o", str(LIB), *map(str, objs), "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


def main() -> int:
    force = "--force" in sys.argv
    build_lib(force=force, verbose=True)
    sys.path.insert(0, str(ROOT))
    from oracle import build as obuild  # the checker, built beside the product

    obuild.build(force=force)
    print("built", LIB)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
