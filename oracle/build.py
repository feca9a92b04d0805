"""Builds the CPU oracle (test infrastructure only) into oracle/liboracle.so.

The oracle is the checker and the timed CPU baseline; the product library never links it.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
OUT = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    deps = [SRC, HERE.parent / "include" / "pmb.h", Path(__file__)]
    if not force and OUT.exists() and all(d.stat().st_mtime <= OUT.stat().st_mtime for d in deps):
        return OUT
    tmp = OUT.with_suffix(".so.tmp")
    cmd = ["g++", "-O3", "-march=x86-64-v2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
