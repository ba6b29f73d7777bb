"""Compile the oracle's C restatement (and the CPU-baseline port) into oracle/liborc.so."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"
SOURCES = ["fgf_oracle.c", "cpu_port.c"]


def build(force: bool = False) -> Path:
    srcs = [HERE / s for s in SOURCES if (HERE / s).exists()]
    deps = srcs + list(HERE.glob("*.h"))
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    cmd = ["gcc", "-O3", "-std=c11", "-shared", "-fPIC", "-pthread", "-o", str(LIB), *map(str, srcs)]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("built", LIB)
