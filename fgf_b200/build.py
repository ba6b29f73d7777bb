"""Build libfgfcuda.so in-tree (sm_100a) and the oracle's C library.

Usage: python -m fgf_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libfgfcuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["kernels.cu", "batch.cu", "api.cpp", "tables.cpp", "serve.cpp"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_lib(force: bool = False, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.hpp")) + [ROOT / "include" / "fgf_cuda.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-cudart", "static", "-Xptxas", "-warn-spills", "-o", str(LIB), *map(str, srcs),
           "-lpthread"]
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
